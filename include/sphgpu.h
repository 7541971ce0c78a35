/*
 * sphgpu.h -- C ABI of the B200 (sm_100a) time-step engine for the multi-phase
 * SPH solver wodexinxin2015/MultiPhase-SPH-Solver.
 *
 * The engine owns one particle system in device memory (structure of arrays,
 * FP64) and runs the reference's per-step particle loop on the GPU.  Every
 * entry point takes plain pointers and sizes; no C++ or torch types cross the
 * boundary.  Return value convention (all int-returning entry points):
 *     0            success
 *     3            a particle left the cell grid       (reference: parttocell)
 *     5            a particle has more than 99 neighbours (partisearching)
 *     >= 100       engine errors (SPHGPU_E_*)
 * These are the integers the reference returns from the methods this layer
 * replaces, so a caller's Err_Deal() keeps working unchanged.
 *
 * Reference interfaces replaced (file:line in the reference project):
 *   clNNPS_Fun::celllist_ini1/ini2/parttocell/partisearching
 *                                         Class_Functions.h:41-59, CPP_3-NNPS.cpp:96-374
 *   clDensity_Fun::density                Class_Functions.h:61-67, CPP_6-density.cpp:11-189
 *   clStraStre_Fun::strain_noreg/eos/strain_to_stress/free_surface_check/
 *                   Stress_eigValue/stress_regu/strain_regu
 *                                         Class_Functions.h:69-82
 *   clInterFor_Fun::cal_permeability/interact1
 *                                         Class_Functions.h:106-119
 *   clAcce_Fun::fluid_acceleration_*, soil_acceleration_noreg,
 *               structure_acceleration_noreg, boundary_moving_stress_effect,
 *               artificial_viscosity      Class_Functions.h:121-150
 *   clVel_Fun::veocity_update/xsph        Class_Functions.h:156-162
 *   clUpdate_Fun::update/timestep         Class_Functions.h:164-169
 *   clBndy_Fun::tmboundary/check_domain   Class_Functions.h:171-185
 *   the step sequence of SPH_Calculation  CPP_1-SPHLoops.cpp:478-775
 */
#ifndef SPHGPU_H_INCLUDED
#define SPHGPU_H_INCLUDED

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPHGPU_ABI_VERSION 1
#define SPHGPU_MAX_NEIGHBORS 99   /* Par_Cell::influ[100] is 1-based: Class_NNPS.h:71 */

/* error codes beyond the reference's own (which are 1..42) */
#define SPHGPU_E_ARG        100   /* bad argument / unknown field name          */
#define SPHGPU_E_CUDA       101   /* a CUDA runtime call failed                 */
#define SPHGPU_E_NODEVICE   102   /* no CUDA device or the kernels failed to load */
#define SPHGPU_E_UNSUPPORTED 103  /* a flag combination this engine does not run */
#define SPHGPU_E_STATE      104   /* call order (e.g. step before upload)        */
#define SPHGPU_E_CHECK      106   /* bounds-checked build (libsphgpu_check.so): an index of the
                                     neighbour search out of range or inconsistent */

/* Para_Fluid, field for field (Class_ParticleProperty.h:107-133). */
typedef struct sphgpu_fluid {
    double vis, vpu, dens, paa0, porosity, fai, c;
    int    bhtype, press_type, acc_type;
    double pre_coe, strain_min;
} sphgpu_fluid;

/* Para_Soil, field for field (Class_ParticleProperty.h:33-105). */
typedef struct sphgpu_soil {
    double e, poi, eps0, dens, damp1, damp2, cop, ramda, kapa, zmf;
    double ann, bnn, beta, sitas, sitar, epsr, epss, sd, sw, kse;
    double c1, c2, c3, fai, c, ocr, sme0, mzm, azm, r0;
    double bl, bz, zet, vpu, porosity, fs, etao, g0, ds, damp_coe;
} sphgpu_soil;

/* Para_Structure (Class_ParticleProperty.h:135-151). */
typedef struct sphgpu_structure {
    double dens, eps0, e, poi, vpu, porosity, cop;
} sphgpu_structure;

/*
 * Run parameters: the union of Para_FL, Para_Pro, Para_Inter, Para_SSInter,
 * Para_Boundary, Para_GF and Cell_Con (Class_Problem.h:10-140,
 * Class_NNPS.h:12-37) that the step loop reads, plus the free-surface
 * thresholds SPH_Calculation keeps as locals (CPP_1-SPHLoops.cpp:81-84).
 */
typedef struct sphgpu_params {
    int    ndim;              /* 2 or 3 */
    int    ntotal;            /* particles */
    /* Para_FL */
    int    fla, fls, flr, fli, flv, fleob, flts, flspv, flknl, flbndy;
    /* Para_Pro */
    int    inip, step_regu, loop, fop;
    double dr, dt;
    double xsph[3];
    double art_vis[3][2];
    double art_stre_coe;
    /* Para_GF */
    double gx, gy, gz;
    /* free surface colour thresholds (input block PR) */
    double threshold_min, threshold_max;
    /* Para_Inter */
    double interc;
    int    permtype;
    double pers, perl, perm;
    /* Para_SSInter */
    int    ss_type;
    double ss_myu, ss_zeta;
    int    ss_acc_type;
    /* Para_Boundary */
    double coe_bndy;
    int    if_cal, if_move;
    double move_vx[3];
    /* Cell_Con: domain box and cell counts (celllist_ini1, CPP_3-NNPS.cpp:96-121) */
    double xmin, xmax, ymin, ymax, zmin, zmax;
    int    cxm, cym, czm, ctotal;
    /* Para_Model / Para_Fluid switches the loop branches on */
    int    flagum;
    double alphats;
    int    water_acc_type;    /* pWater[0].acc_type: 0 plus-form, 1 minus-form */
    int    air_acc_type;      /* pAir->acc_type */
    sphgpu_structure structure;
} sphgpu_params;

typedef struct sphgpu_ctx sphgpu_ctx;

/* Library / device. */
int         sphgpu_abi_version(void);
int         sphgpu_device_count(void);
const char* sphgpu_error_string(int code);

/*
 * Context lifetime.  sphgpu_create copies *params, allocates every device
 * buffer for params->ntotal particles and params->ctotal cells on `device`,
 * and creates the context's CUDA stream.  Returns NULL on failure; the reason
 * is available from sphgpu_last_create_error().
 */
sphgpu_ctx* sphgpu_create(const sphgpu_params* params, int device);
int         sphgpu_last_create_error(void);
void        sphgpu_destroy(sphgpu_ctx* ctx);
int         sphgpu_get_params(const sphgpu_ctx* ctx, sphgpu_params* out);

/*
 * Batched context: many instances of the step (Monte Carlo realisations,
 * slope geometries of uneven particle counts) in one particle system, each
 * step running every instance in the same kernel launches (one CUDA graph per
 * step), driven by a per-instance table of particle offsets and cell grids.
 * The reference runs each instance as a project of its own (CPP_0-main.cpp,
 * one SPH_Calculation per directory); here instance q holds particles
 * [first, first + count) of the context, in the order of its own Particle
 * array, and the cell grid its Cell_Con gives (celllist_ini1,
 * CPP_3-NNPS.cpp:96-121); the instances follow one another (first of the
 * first is 0, each next starts where the last ends).  `shared` holds every
 * other parameter, the same for all instances (its ntotal and grid members
 * are ignored).  Each instance evolves exactly as a context of its own would:
 * its neighbours come from its own cells only, and every absolute particle
 * index the reference uses (check_domain's first moving wall, tm_boundary's
 * particle 0) is taken within the instance.  Fields, records and neighbour
 * lists are indexed by the context's particle index.  sphgpu_update_params
 * is not available for a batched context.
 */
typedef struct sphgpu_instance {
    int    first, count;
    double xmin, xmax, ymin, ymax, zmin, zmax;    /* Cell_Con domain box */
    int    cxm, cym, czm, ctotal;                 /* Cell_Con cell counts */
} sphgpu_instance;
sphgpu_ctx* sphgpu_create_batched(const sphgpu_params* shared, const sphgpu_instance* inst, int ninst,
                                  int device);
int         sphgpu_instance_count(const sphgpu_ctx* ctx);
/* Current step counter l (Para_Pro::l); starts at 1 like the reference. */
int         sphgpu_get_step(const sphgpu_ctx* ctx);
int         sphgpu_set_step(sphgpu_ctx* ctx, int l);

/*
 * Precision form of the step (the reference has one, FP64: every method of
 * clDensity_Fun / clStraStre_Fun / clAcce_Fun / clVel_Fun, Class_Functions.h:61-162).
 *   SPHGPU_PREC_FP64       the drop-in: the reference's FP64 arithmetic, operation
 *                          for operation (the default)
 *   SPHGPU_PREC_FP32_BULK  pair arithmetic of the neighbour passes (kernel values
 *                          and gradients, pair terms and their sums) in FP32 with
 *                          Kahan-compensated sums; positions, velocities, densities,
 *                          stresses, time integration, the constitutive update and
 *                          the neighbour search stay FP64, so neighbour lists are
 *                          identical in both forms
 * May be switched between steps; the state carries over.
 */
#define SPHGPU_PREC_FP64      0
#define SPHGPU_PREC_FP32_BULK 1
int         sphgpu_set_precision(sphgpu_ctx* ctx, int mode);
int         sphgpu_get_precision(const sphgpu_ctx* ctx);

/*
 * Field transfer, structure of arrays.  `name` is a Particle member
 * (Class_particle.h:13-103): "xp", "vx", "sig", "rho", "type", ...
 * sphgpu_field_info reports the component count and element type
 * (0 = double, 1 = int32).  Host layout is particle-major
 * (host[i * ncomp + k]), as the members are laid out in Particle.
 */
int sphgpu_field_info(const char* name, int* ncomp, int* elem_type);
int sphgpu_set_field(sphgpu_ctx* ctx, const char* name, const void* host, size_t count);
int sphgpu_get_field(sphgpu_ctx* ctx, const char* name, void* host, size_t count);

/*
 * Per-particle material records, as SPH_Calculation keeps them
 * (pVFluid / pParti_ConsPara, CPP_1-SPHLoops.cpp:371-372; filled by
 * setting_vis_cons, CPP_2-initialf.cpp:1021-1058).  Either pointer may be
 * NULL (the corresponding records stay zero).  Call it after the particles'
 * matype is set: the members only unsaturated (matype % 10 == 3) and
 * fractional-order (8) Cam-clay and the saturation pass (flagum == 1) read
 * are uploaded when such particles are present, and a step that needs them
 * without them returns SPHGPU_E_STATE.
 */
int sphgpu_set_materials(sphgpu_ctx* ctx, const sphgpu_fluid* fluid,
                         const sphgpu_soil* soil, int n);

/*
 * Whole-record transfer in the reference's Particle layout
 * (Class_particle.h:13-103, 1064 bytes per particle, 8-byte aligned doubles,
 * four trailing ints).  `stride` is sizeof(Particle) on the caller's side and
 * must be >= 1064.  Download writes only the members the device owns.
 */
int sphgpu_upload_particles(sphgpu_ctx* ctx, const void* particles, int n, size_t stride);
int sphgpu_download_particles(sphgpu_ctx* ctx, void* particles, int n, size_t stride);
/* Byte offset and component count of a Particle member in the record layout
 * the two calls above use; returns SPHGPU_E_ARG for members they skip. */
int sphgpu_particle_layout(const char* name, size_t* offset, int* ncomp);

/*
 * One or more complete time steps: the body of the main loop of
 * SPH_Calculation (CPP_1-SPHLoops.cpp:523-753) for steps l, l+1, ...
 * Host-side work the loop interleaves (rain, excavation, output) is the
 * caller's.  Returns 0 or the first error code raised; on error the step
 * counter stays at the failing step.
 */
int sphgpu_step(sphgpu_ctx* ctx, int nsteps);

/*
 * Step l in the reference's method granularity, for the C++ shim classes that
 * keep SPH_Calculation's own loop (CPP_1-SPHLoops.cpp:523-753) as the caller:
 *   sphgpu_parttocell      clNNPS_Fun::parttocell (CPP_3-NNPS.cpp:175-263):
 *                          cell keys, the radix sort in Binary_Sort's order and
 *                          the cell ranges; returns 0 or 3
 *   sphgpu_partisearching  clNNPS_Fun::partisearching (CPP_3-NNPS.cpp:265-374):
 *                          the neighbour lists and their kernel values; runs
 *                          parttocell first if the step has not; returns 0 or 5
 *   sphgpu_update          every method SPH_Calculation calls after
 *                          partisearching, through clUpdate_Fun::update
 *                          (kernel_gradient_correction, density, strain_noreg,
 *                          strain_regu, saturation, cal_permeability, eos,
 *                          strain_to_stress, stress_regu, free_surface_check,
 *                          Stress_eigValue, the clAcce_Fun accelerations,
 *                          artificial viscosity and stress, the wall stresses,
 *                          coupled_Water_Soil_Structure, interact1/2/3,
 *                          interaction_ss_*, soil_damping_geostress,
 *                          boundary_free_solid, veocity_update, xsph, the wall
 *                          treatments of clBndy_Fun, check_domain, update): the
 *                          engine fuses these methods into passes that cross the
 *                          methods' boundaries (the local equation of state
 *                          runs with the Shepard filter, seven momentum methods
 *                          share one neighbour pass), so they run together
 *                          when the step completes; advances l.  Runs the
 *                          search first if the step has not.
 * The results equal sphgpu_step's.  sphgpu_parttocell on a step whose cell
 * lists are built returns SPHGPU_E_STATE; sphgpu_step completes a step these
 * entries began before it runs its own.
 */
int sphgpu_parttocell(sphgpu_ctx* ctx);
int sphgpu_partisearching(sphgpu_ctx* ctx);
int sphgpu_update(sphgpu_ctx* ctx);

/*
 * Replace the run flags and parameters of a context between steps (a caller
 * that learns them method by method, as the shim classes do).  The particle
 * count, dimension and cell grid must be those the context was created with
 * (else SPHGPU_E_ARG); buffers new flags need are allocated here.
 */
int sphgpu_update_params(sphgpu_ctx* ctx, const sphgpu_params* params);

/*
 * The NNPS stage alone (parttocell + partisearching for step l), leaving the
 * neighbour lists on the device; ninflu[n] and influ[n * 100] (1-based slots
 * 1..ninflu, as Par_Cell::influ) are copied out if non-NULL.
 */
int sphgpu_nnps(sphgpu_ctx* ctx, int* ninflu, int* influ);

/*
 * Adaptive time step (an addition of this library: the reference's dt is
 * constant, clUpdate_Fun::timestep, CPP_12-2-dt.cpp:13-20).  With cfl > 0 the
 * last kernels of every step reduce, over the water, soil, air and structure
 * particles, min(cfl h / (c + |v|), cfl_force sqrt(h / |a|)) -- c the sound
 * speed of the particle's material (Para_Fluid / Para_Soil / Para_Structure
 * vpu), v and a its velocity and acceleration after the update -- with warp
 * shuffles on the device, and the next step runs with that dt, capped at the
 * input dt (no host round trip: the steps stay in their CUDA graphs).  The
 * first step after the call uses the input dt.  cfl <= 0 turns it off, the
 * default; every parity statement of this library is for the constant dt.
 * sphgpu_get_dt reads the dt the next step will use.
 */
int sphgpu_set_cfl(sphgpu_ctx* ctx, double cfl, double cfl_force);
int sphgpu_get_dt(sphgpu_ctx* ctx, double* dt);

/*
 * Re-sorted state (an addition of this library; the reference keeps its
 * particle array in input order and only sorts an index list, Binary_Sort,
 * CPP_3-NNPS.cpp:561-630).  With every_steps > 0, sphgpu_step and
 * sphgpu_step_profiled gather the whole particle state on the device into a
 * spatial order -- by type and material, then rows of a lattice of spacing dr
 * over the grid (over each batched instance's own grid) along its longest
 * axis -- before the next step and then every every_steps steps, so the
 * neighbour gathers of the passes read nearby records whatever order the
 * caller's particles came in or have mixed into.  Every result stays the one
 * of the caller's order, bit for bit: the device keeps the map between the
 * orders, and the passes whose result
 * depends on the particle numbering (the search's order inside a cell, the
 * rain rows, check_domain's first wall, tm_boundary's default wall, the order
 * of a structure particle's contact reactions) go through it.  Every call that
 * exchanges per-particle data with the host, or runs part of a step through
 * the method entries, first gathers the state back into the caller's order
 * (on the device; the result-file snapshot of sphgpu_output_step writes its
 * rows through the map instead).  0 (the default) keeps the caller's order.
 * sphgpu_get_order copies the map out: i2o[i] = the caller's index of the
 * particle held at i (N ints).  sphgpu_last_reorder_ms is the device time the
 * re-sorts of the last sphgpu_step_profiled call took.
 */
int sphgpu_set_reorder(sphgpu_ctx* ctx, int every_steps);
int sphgpu_get_reorder(const sphgpu_ctx* ctx);
int sphgpu_get_order(sphgpu_ctx* ctx, int* i2o);
double sphgpu_last_reorder_ms(const sphgpu_ctx* ctx);
/*
 * Chooses between the two by timing (the steps are real steps of the run):
 * `steps` steps in the caller's order, then a re-sort and `steps` more, and
 * keeps re-sorting every `every` steps only when the re-sorted steps, with the
 * time of a further re-sort (of the re-sorted state, as every re-sort after
 * the first is) charged per `every` steps, are more than 3% faster.  *chosen
 * is the interval set (every or 0); ms[0..2], if non-NULL, the caller's-order
 * step, the re-sorted step and the re-sort's share per step (device ms, the
 * per-stage sums of sphgpu_step_profiled).  With 0 chosen the state is back in
 * the caller's order.
 */
int sphgpu_autotune_reorder(sphgpu_ctx* ctx, int steps, int every, int* chosen, double* ms);

/*
 * Rainfall (flr == 1): the reference's Para_Rain (Class_Problem.h) as its
 * input block RP sets it, with nrain the number of rain particles still
 * waiting (type 7, etype 1; input_par counts them, CPP_2-initialf.cpp:979-
 * 1017).  The rain particles sit at the end of the particle array, row after
 * row in the order they fall.  Every lp steps (rainini, CPP_15-1-rain.cpp:
 * 11-23: lp = (loop - inip) / (nrain / nhor + 1)) the top of the step
 * releases the next row (rainpro, :43-85), and after the update water beyond
 * the domain's x ends is taken out (partidel, CPP_15-2-partidel.cpp:19-58);
 * both run on the device inside the step's CUDA graph, with no host round
 * trip.  rtype 1 (rain) is supported; 2-4 (water-level lowering, cement
 * injection) return SPHGPU_E_UNSUPPORTED.  sphgpu_get_rain reports nrain as
 * the steps have left it.  A context created with flr == 1 steps only after
 * sphgpu_set_rain (SPHGPU_E_STATE before).
 */
typedef struct sphgpu_rain {
    int    rtype, nrain, nhor;
    double press_factor, drop_velocity;
} sphgpu_rain;
int sphgpu_set_rain(sphgpu_ctx* ctx, const sphgpu_rain* rain);
int sphgpu_get_rain(sphgpu_ctx* ctx, sphgpu_rain* rain);

/*
 * Checkpoint and restart (the reference has none: a run restarts only from
 * its input deck).  sphgpu_checkpoint_save writes, between steps, the step
 * counter, every device-owned Particle member, the material records, the
 * precision form, the rain and adaptive-step settings, and the device state
 * outside Particle that the next step reads (the walls' per-phase virtual
 * velocities and stresses of flbndy 2-4 / 13 / 14, the range of the cell
 * ctotal that the reference never resets, the rain and time-step words).
 * sphgpu_checkpoint_load restores it into a context created with the same
 * parameters; the run then continues bit for bit as it would have.  Returns
 * 0, SPHGPU_E_ARG (unreadable file or another particle count or grid), or an
 * engine code.
 */
int sphgpu_checkpoint_save(sphgpu_ctx* ctx, const char* path);
int sphgpu_checkpoint_load(sphgpu_ctx* ctx, const char* path);

/*
 * Result files, written while the steps go on (the reference writes them on
 * the host between steps, clOutput_Fun::output_total, CPP_14-2-output.cpp:
 * 15-136).  sphgpu_output_total takes a snapshot of the state after the last
 * completed step l on the step stream (the next step starts after it), copies
 * it to pinned host memory on a stream of its own and writes
 * dir/data-<l, 10 digits>.odb from a host thread, in output_total's format
 * byte for byte (rows formatted on several threads), while later steps run.
 * Two files may be in flight; a third call waits for the older.
 * sphgpu_output_wait waits for every file and returns the first error of
 * their writing (0 if none).  The snapshot memory (two buffers of 49 doubles
 * per particle on the device and in pinned host memory) is allocated at the
 * first call.
 */
int sphgpu_output_total(sphgpu_ctx* ctx, const char* dir);
int sphgpu_output_wait(sphgpu_ctx* ctx);
/*
 * The other result files of SPH_Calculation's output steps
 * (CPP_1-SPHLoops.cpp:761-780), from the same snapshot: sphgpu_output_step
 * writes the files `what` selects, the data-*.odb of output_total included,
 * and appends to the run's files in call order.  sphgpu_output_begin creates
 * dir's "Flowing distance.dat", Total_Force.dat and AVS_MGF.mgf (with the AVS
 * header and the frame count loop / fop) as SPH_Calculation opens them
 * before its loop (:185-230, 452-453).
 */
#define SPHGPU_OUT_ODB      1   /* data-<l>.odb (output_total, CPP_14-2-output.cpp:15-136) */
#define SPHGPU_OUT_FLOWDIST 2   /* each phase's extent, appended to "Flowing distance.dat" (output_flowdist, :222-320) */
#define SPHGPU_OUT_IMPACT   4   /* Impact-force<l>.inp and a Total_Force.dat line (output_impact, :139-220) */
#define SPHGPU_OUT_MGF      8   /* a frame appended to AVS_MGF.mgf (mgf, CPP_14-1-outmgf.cpp:12-104) */
int sphgpu_output_begin(sphgpu_ctx* ctx, const char* dir);
int sphgpu_output_step(sphgpu_ctx* ctx, const char* dir, int what);

/* Block until the context's stream is idle; returns the sticky error, if any. */
int sphgpu_synchronize(sphgpu_ctx* ctx);

/*
 * Timing: CUDA-event duration of the last sphgpu_step call (milliseconds), and
 * the number of kernels that call launched.
 */
double sphgpu_last_step_ms(const sphgpu_ctx* ctx);
long   sphgpu_last_step_launches(const sphgpu_ctx* ctx);

/*
 * Launch shapes and their autotuner (no counterpart in the reference, whose
 * OpenMP loops take their thread count from the input deck).  Each of the
 * SPHGPU_TUNE_PASSES neighbour passes -- the search scan, its resolve pass,
 * the pair records, density, Shepard + EOS, strain, the constitutive update,
 * the two momentum stages, XSPH + update, in that order -- runs one particle
 * per thread with 32 to 128 threads per block (a multiple of 32).
 * sphgpu_set_launch / sphgpu_get_launch set and read those sizes;
 * sphgpu_autotune runs `steps` steps of the run with each of 32, 64, 96 and
 * 128 threads per block, times every pass with CUDA events, and keeps for
 * each pass the fastest, a shape other than 128 only when it is more than 3%
 * faster (the spread of the timings).  The steps it runs are steps of the
 * run: a launch shape changes no result, bit for bit.  With cache_path the
 * choice is kept in that text file under a key of the GPU model and the
 * run's shape (dimension, particle count, wall, drag and contact types,
 * precision form, instances), and a later call with the same key applies it
 * without measuring.  table, if non-NULL, receives the mean ms per step of
 * each pass for each candidate (4 x SPHGPU_TUNE_PASSES, candidate-major).
 */
#define SPHGPU_TUNE_PASSES 10
int sphgpu_set_launch(sphgpu_ctx* ctx, const int* threads_per_block, int n);
int sphgpu_get_launch(const sphgpu_ctx* ctx, int* threads_per_block, int n);
int sphgpu_autotune(sphgpu_ctx* ctx, int steps, const char* cache_path, double* table);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work after the engine's. */
void*  sphgpu_stream(sphgpu_ctx* ctx);

/*
 * Stage-level profile: runs nsteps like sphgpu_step, but launching each stage
 * directly on the context's stream with a CUDA event between consecutive
 * stages, and adds each stage's duration (ms, summed over the steps) to
 * stage_ms[0 .. sphgpu_stage_count()-1].  Stage k is named by
 * sphgpu_stage_name(k) (the kernel names, plus "radix_sort").
 */
int         sphgpu_stage_count(void);
const char* sphgpu_stage_name(int k);
int         sphgpu_step_profiled(sphgpu_ctx* ctx, int nsteps, double* stage_ms);

/*
 * Vibration loading (flv 1 and 2): Para_Vibra (Class_Problem.h:133-149) as
 * initial_pro reads its VL block (ttime nsteps / sttime edtime,
 * CPP_2-initialf.cpp:250-270) and initial_vib reads vibra.dat (nsteps rows of
 * three loads, CPP_2-initialf.cpp:292-320).  With flv 1 the walls of matype 3
 * and 5 take the load of the step's time as their acceleration
 * (vibration_acceleration, CPP_9-1-acceleration_vibration.cpp:10-78), with
 * flv 2 the walls of matype 4 and 5 take it as their velocity
 * (vibration_velocity, :80-160); with either, the soil and structure
 * particles are damped by soil_damping_vibration (:162-224, damp1 + damp2
 * sqrt(stiffness / rho h^2) from the soil record) and the soil feels the
 * free-field particles (free_field_solid, CPP_19-FreeFieldParticles.cpp and
 * CPP_19-FreeFieldParticles_soil.cpp: soil of matype >= 50 and walls of
 * matype 5, permtype the wave direction).  A context with flv >= 1 steps
 * only after this call.  Returns 0, 7 (nsteps < 1, the reference's error),
 * SPHGPU_E_ARG (no loads, or ttime not positive), SPHGPU_E_STATE (flv 0).
 * sphgpu_checkpoint_save keeps the table.
 */
typedef struct sphgpu_vibration {
    double ttime;                /* one period */
    int    nsteps;               /* load entries per period */
    double sttime, edtime;       /* the loads apply for sttime <= t <= edtime */
} sphgpu_vibration;

int sphgpu_set_vibration(sphgpu_ctx* ctx, const sphgpu_vibration* vib, const double* loads);

/*
 * Karhunen-Loeve random fields (flspv 1 and 2): the reference's
 * clFSpatialVariability_Fun::SpatialVariables_Generate_2D / _3D and
 * SpatialVariables_Generate_2D_corr / _3D_corr
 * (Class_spatial_variability.h:79-86, CPP_17-1_K-L_expansion_non.cpp:62-272,
 * CPP_17-2_K-L_expansion_corr.cpp:55-473).
 *
 * sphgpu_kl_field is Para_SpatialVariability (Class_spatial_variability.h:46-66)
 * without its derived half extents; `no` selects the member written:
 * 0 soil fai, 1 soil c, 2 soil cop, 3 soil ds (type-2 particles), 4 fluid fai,
 * 5 fluid c (type-1 particles).  sphgpu_kl_domain holds the Cell_Con members
 * the generators read (Class_NNPS.h): the extents of the non-boundary
 * particles (xmin_nb .. zmax_nb) and soil_max / water_max as input_par stores
 * them (CPP_2-initialf.cpp:954-961).
 *
 * The reference draws the standard normals from a time-seeded generator
 * (generate_SND, CPP_17-1:24-33); here the caller passes them: xi holds K
 * values per field (sphgpu_kl_generate) or K x 2 values per correlated pair
 * (sphgpu_kl_generate_corr, the uu_cfai matrix of CPP_17-2:121).  K is the
 * number of terms, the reference's klterm (200); other K are accepted.
 * The fields are written into the context's material records for the
 * particles each field covers (sphgpu_set_materials must have been called)
 * and the constants the step derives from them are evaluated again; out, if
 * non-NULL, receives nfields x ntotal values (NaN where a field writes none).
 * Returns 0, 13 (a zero half extent, as the reference), 14 (a distribution
 * type other than 1 or 2), or an engine code.
 */
typedef struct sphgpu_kl_field {
    int    no;                /* member written (above) */
    int    type;              /* 1 normal, 2 lognormal */
    double mean_value, sd_value;
    double rl_value[3];       /* correlation lengths */
    double coe_depth;         /* mean + (top - y) * coe_depth */
} sphgpu_kl_field;

typedef struct sphgpu_kl_domain {
    double xmin_nb, xmax_nb, ymin_nb, ymax_nb, zmin_nb, zmax_nb;
    double soil_max[3], water_max[3];
} sphgpu_kl_domain;

int sphgpu_kl_generate(sphgpu_ctx* ctx, const sphgpu_kl_domain* dom, const sphgpu_kl_field* fields, int nfields,
                       const double* xi, int K, double* out);
/* Correlated friction / cohesion (flspv 2): pairs[0] is the friction field
 * (no 0 or 4) and pairs[1] the cohesion field (no 1 or 5) of one phase;
 * coe_frict_cohesion is Flag_SpatialVariability::coe_frict_cohesion. */
int sphgpu_kl_generate_corr(sphgpu_ctx* ctx, const sphgpu_kl_domain* dom, const sphgpu_kl_field pair[2],
                            double coe_frict_cohesion, const double* u2, int K, double* out);

/*
 * Correlation-matrix random fields: the reference's
 * clFSpatialVariability_Fun::nonstationary_random_2D / _3D (flspv 3,
 * Class_spatial_variability.h:92-103, CPP_17-3-Nonstationary-RF.cpp:76-458,
 * 460-849), nonstationary_correlated_random_2D / _3D (flspv 4,
 * CPP_17-5-Nonstationary-Correlated-RF.cpp:87-406, 409-735) and
 * random_variable_generate (flspv 5, CPP_17-5:738-863).
 *
 * The non-boundary box (sphgpu_kl_domain), widened by 10% per side, is cut
 * into cells of cell_ndx particle spacings; the correlation matrix of the
 * cell centres is factored (Cholesky, the diagonal's radicand floored at
 * 1e-6), multiplied by one standard normal per cell, and every particle of a
 * cell takes the cell's value (2-D: water and soil particles are placed in
 * cells; 3-D: every particle).  sphgpu_rf_flags holds the
 * Flag_SpatialVariability members the generators read
 * (Class_spatial_variability.h:9-36).
 *
 * The reference draws the normals from a time-seeded generator
 * (generate_SND, CPP_17-3:31-41); here the caller passes them:
 * sphgpu_rf_cells gives the number of cells C, and zeta holds C values per
 * field in the reference's cell order (x fastest, then y, then z).  The
 * fields are written into the material records (sphgpu_set_materials must
 * have been called) as sphgpu_kl_generate writes them; out, if non-NULL,
 * receives nfields x ntotal values (NaN where a field writes none).
 * Returns 0, 41 (no cells, or 15,000 or more), 42 (a cell holding more than
 * 39 particles), SPHGPU_E_ARG (a particle outside the cells, where the
 * reference would index past its cell array; or ncell is not C),
 * SPHGPU_E_UNSUPPORTED for a batched context, or an engine code.
 */
typedef struct sphgpu_rf_flags {
    double cell_ndx;             /* cell edge in particle spacings */
    int    flag_auto;            /* 1 exponential, 2 Gaussian, 3 rotated exponential */
    double beta, beta_1;         /* rotation angles (flag_auto 3), degrees */
    double coe_frict_cohesion;   /* correlation of friction and cohesion (flspv 4 and 5) */
} sphgpu_rf_flags;

int sphgpu_rf_cells(sphgpu_ctx* ctx, const sphgpu_kl_domain* dom, const sphgpu_rf_flags* flags, int* ncell);
/* flspv 3: fields in the caller's order, each with its own factor (as the
 * reference, which factors again per field; consecutive fields of equal
 * correlation lengths share one here) */
int sphgpu_rf_generate(sphgpu_ctx* ctx, const sphgpu_kl_domain* dom, const sphgpu_kl_field* fields, int nfields,
                       const sphgpu_rf_flags* flags, const double* zeta, int ncell, double* out);
/* flspv 4: pair[0] the friction field (no 0 or 4), pair[1] the cohesion field
 * (no 1 or 5) of one phase; u2 holds ncell x 2 normals (the reference's
 * vec_zeta_1), correlated through the 2 x 2 factor of coe_frict_cohesion.
 * Both members use the friction field's correlation lengths and distribution
 * type; out receives 2 x ntotal values. */
int sphgpu_rf_generate_corr(sphgpu_ctx* ctx, const sphgpu_kl_domain* dom, const sphgpu_kl_field pair[2],
                            const sphgpu_rf_flags* flags, const double* u2, int ncell, double* out);
/* flspv 5: one correlated pair of random variables for the whole phase from
 * the two normals u2; out receives the friction and cohesion values. */
int sphgpu_rv_generate_corr(sphgpu_ctx* ctx, const sphgpu_kl_field pair[2], double coe_frict_cohesion,
                            const double u2[2], double out[2]);

/*
 * K-L fields of a batched context: one field per instance, each over the
 * instance's own particles with its own domain doms[q] and its own standard
 * normals xi[q * K .. q * K + K - 1] (what sphgpu_kl_generate does for one
 * system, for every instance in one call, with one update of the material
 * records at the end).  out, if non-NULL, receives ntotal values.
 */
int sphgpu_kl_generate_batched(sphgpu_ctx* ctx, const sphgpu_kl_domain* doms, const sphgpu_kl_field* field,
                               const double* xi, int K, double* out);

/*
 * Batched synthesis of R realisations of one field on the context's particles
 * (the Monte Carlo use of the generator above: R runs of
 * SpatialVariables_Generate_2D / _3D on one geometry, each with its own
 * normals).  xi: R x K standard normals (host); d_out: a DEVICE buffer of
 * R x ntotal floats receiving field value [r * ntotal + i] (NaN where the
 * field writes none).  The sum over the K terms runs on the tensor cores as
 * an FP32-accurate product of TF32 operand halves; values agree with the FP64
 * generator to FP32 rounding.  R must be a multiple of 16 and K of 8.
 * kernel_ms, if non-NULL, receives the device time of the synthesis kernels.
 * Returns 0, 13, 14, SPHGPU_E_ARG, or SPHGPU_E_KL_TIMEOUT if a tensor-core
 * completion wait expired (the outputs are then incomplete).
 */
#define SPHGPU_E_KL_TIMEOUT 105
/*
 * Self-test of the synthesis kernel's failure path (no counterpart in the
 * reference): one CTA of the kernel takes its tensor memory and waits
 * budget_cycles SM clocks on a completion barrier that nothing will signal,
 * before it has issued any MMA; the wait must expire, the kernel must record
 * the timeout and release the memory, and the context stays usable.  Returns
 * SPHGPU_E_KL_TIMEOUT when that happened (the expected result).
 */
int sphgpu_kl_wait_check(sphgpu_ctx* ctx, long long budget_cycles);

/*
 * The device's FP64 and FP32 multiply-add rates in TFLOP/s (two flops per
 * fused multiply-add), measured by a kernel of independent multiply-add
 * chains on every SM (no counterpart in the reference): the denominators of
 * the compute side of the step's roofline.  Takes a few milliseconds.
 */
int sphgpu_pipe_peaks(int device, double* fp64_tflops, double* fp32_tflops);
int sphgpu_kl_synthesize(sphgpu_ctx* ctx, const sphgpu_kl_domain* dom, const sphgpu_kl_field* field,
                         const double* xi, int R, int K, float* d_out, double* kernel_ms);

/*
 * Neighbour search that allocates no device memory (no counterpart in the
 * reference: an addition of this library).
 *
 * For callers that cannot call cudaMalloc where they need neighbour lists --
 * code under a device-memory pool or budget that forbids new allocations, a
 * real-time loop that must stay out of the driver's allocator, or a host
 * application that owns every device buffer and only lends pointers.  The
 * caller passes device pointers: d_xp (n * 3 doubles, particle-major, as
 * Particle::xp), d_hl (n doubles), d_type (n ints) in, and d_ninflu (n ints)
 * and d_influ (n * 100 ints, Par_Cell::influ layout: slots 1..ninflu) out;
 * `grid` supplies ndim, dr, xmin/ymin/zmin and cxm/cym/czm/ctotal.  The
 * result equals what sphgpu_nnps returns on the same positions for the first
 * search after the particles are loaded (parttocell + partisearching,
 * CPP_3-NNPS.cpp:175-374).  The reference, and the context engine, carry the
 * cell range of the extra cell ctotal over from step to step
 * (CPP_3-NNPS.cpp:196-201); each call here starts it afresh.
 *
 * Every intermediate lives in one fixed device array of
 * sphgpu_nnps_noalloc_scratch_bytes() bytes inside the library, held by each
 * GPU that loads the library until the process exits; n is limited to
 * SPHGPU_NOALLOC_MAX_PARTICLES and ctotal to SPHGPU_NOALLOC_MAX_CELLS (larger
 * sizes return SPHGPU_E_ARG).  The first call on a device looks the array up
 * with that device current and keeps it for the rest of the process; make it
 * before any stream capture, and do not call the search again on a device the
 * process has reset (cudaDeviceReset discards the array).  All calls on
 * a device share the array: calls that overlap on the GPU race and must not
 * be issued.  The call runs on `stream` (a cudaStream_t, NULL for the default
 * stream) and waits for that stream, so it is synchronous and cannot be
 * captured into a CUDA graph.  Returns 0, 3 (a particle outside the grid; the
 * outputs are not written), 5 (more than 99 neighbours: every count in
 * d_ninflu is written, lists hold their first 99 slots) or SPHGPU_E_CUDA
 * (also when an error of the caller's earlier work is pending; it is left
 * pending and nothing is launched).
 */
#define SPHGPU_NOALLOC_MAX_PARTICLES 65536
#define SPHGPU_NOALLOC_MAX_CELLS     262144
int    sphgpu_nnps_noalloc(const sphgpu_params* grid, int n, const double* d_xp, const double* d_hl,
                           const int* d_type, int* d_ninflu, int* d_influ, void* stream);
size_t sphgpu_nnps_noalloc_scratch_bytes(void);

#ifdef __cplusplus
}
#endif

#endif /* SPHGPU_H_INCLUDED */
