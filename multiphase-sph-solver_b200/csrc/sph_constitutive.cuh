// sph_constitutive.cuh -- per-particle constitutive arithmetic of the step
// (CPP_8-1-consfactor.cpp, CPP_7-2-constitutive.cpp, Class_particle.cpp,
// CPP_7-1-strain.cpp), in the reference's operation order.
#pragma once


__device__ __forceinline__ void jaumann(double ds[6], const double s[6], const double we[9])
{
#define WE(a, b) we[(a) * 3 + (b)]
    ds[0] = ds[0] + (WE(0, 0) * s[0] + WE(0, 1) * s[3] + WE(0, 2) * s[5]) - (s[0] * WE(0, 0) + s[3] * WE(1, 0) + s[5] * WE(2, 0));
    ds[1] = ds[1] + (WE(1, 0) * s[3] + WE(1, 1) * s[1] + WE(1, 2) * s[4]) - (s[3] * WE(0, 1) + s[1] * WE(1, 1) + s[4] * WE(2, 1));
    ds[2] = ds[2] + (WE(2, 0) * s[5] + WE(2, 1) * s[4] + WE(2, 2) * s[2]) - (s[5] * WE(0, 2) + s[4] * WE(1, 2) + s[2] * WE(2, 2));
    ds[3] = ds[3] + (WE(0, 0) * s[3] + WE(0, 1) * s[1] + WE(0, 2) * s[4]) - (s[0] * WE(0, 1) + s[3] * WE(1, 1) + s[5] * WE(2, 1));
    ds[4] = ds[4] + (WE(1, 0) * s[5] + WE(1, 1) * s[4] + WE(1, 2) * s[2]) - (s[3] * WE(0, 2) + s[1] * WE(1, 2) + s[4] * WE(2, 2));
    ds[5] = ds[5] + (WE(0, 0) * s[5] + WE(0, 1) * s[4] + WE(0, 2) * s[2]) - (s[0] * WE(0, 2) + s[3] * WE(1, 2) + s[5] * WE(2, 2));
#undef WE
}

// elastic D (only its nonzero pattern is kept: dlam, dmu) -- elastic(),
// dpmodel1(), dpmodel_bui() share it (:17-59, :301-334, :468-501)
// (elastic_plastic, :618-660, takes the mean stress with third = 0.333333333)
// The elastic modulus: the material's E, or 3 (1 - 2 nu) (1 + e0) |p| / kappa
// when E <= 1 (p = mean compression, at least 1).
__device__ __forceinline__ double elastic_e0(const double s[6], double E, double poi, double eps0, double kapa,
                                             double* sm_out, double third = 0.3333333333)
{
    double sm = (-s[0] + -s[1] + -s[2]) * third;
    if (sm < 1.0) sm = 1.0;
    double e0;
    if (E > 1.0) e0 = E;
    else e0 = 3 * (1 - 2 * poi) * (1 + eps0) * fabs(sm) / kapa;
    *sm_out = sm;
    return e0;
}

__device__ __forceinline__ void elastic_consts(const double s[6], double E, double poi, double eps0, double kapa,
                                               double* dlam, double* dmu, double* sm_out,
                                               double third = 0.3333333333)
{
    double sm;
    const double e0 = elastic_e0(s, E, poi, eps0, kapa, &sm, third);
    *dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
    *dmu = e0 * 0.5 / (1.0 + poi);
    *sm_out = sm;
}

// dsig += D deps, in the reference's dept[ki][kj] * deps[kj] loop order over a
// dense 6x6 with the zero entries included (0 * x terms keep signed-zero and
// NaN behaviour identical).
__device__ __forceinline__ void add_dense(double ds[6], const double D[6][6], const double de[6])
{
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) ds[a] += D[a][b] * de[b];
}

__device__ __forceinline__ void fill_elastic(double D[6][6], double dlam, double dmu)
{
    const double dmu2 = dmu * 2.0;
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) D[a][b] = 0.0;
    D[0][0] = dlam + dmu2; D[1][1] = dlam + dmu2; D[2][2] = dlam + dmu2;
    D[0][1] = dlam; D[0][2] = dlam; D[1][0] = dlam;
    D[1][2] = dlam; D[2][0] = dlam; D[2][1] = dlam;
    D[3][3] = dmu; D[4][4] = dmu; D[5][5] = dmu;
}

// Drucker-Prager continuum tangent (dpmodel1 / dpmodel_bui, :284-448 /
// :451-615) and, with MC = true, the Mohr-Coulomb form of elastic_plastic
// (:618-777: plastic potential without dilatancy and no hardening term in
// the denominator).  yalf, ykap, yalf_dil are the material constants the
// reference evaluates with atan/tan/sin/cos each call; they are evaluated once
// per particle by the host with the same libm calls.
template <bool MC = false>
__device__ __forceinline__ void dp_tangent(double D[6][6], double adps[6], const double s[6], const double de[6],
                                           double dlam, double dmu, double sm,
                                           double yalf, double ykap, double yalf_dil)
{
    const double dmu2 = dmu * 2.0;
    double sig0 = -s[0], sig1 = -s[1], sig2 = -s[2];
    double dx = sig0 - sm, dy = sig1 - sm, dz = sig2 - sm;
    double dxy = -s[3], dyz = -s[4], dzx = -s[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double sj = sqrt(sjj);
    if ((sj - yalf * sm * 3.0 - ykap) >= 0.0) {
        double f11 = -yalf + dx / sj * 0.5, f22 = -yalf + dy / sj * 0.5, f33 = -yalf + dz / sj * 0.5;
        double f12 = dxy / sj * 0.5, f23 = dyz / sj * 0.5, f31 = dzx / sj * 0.5;
        double fkk = f11 + f22 + f33;
        double g11 = MC ? dx / sj * 0.5 : -yalf_dil + dx / sj * 0.5;
        double g22 = MC ? dy / sj * 0.5 : -yalf_dil + dy / sj * 0.5;
        double g33 = MC ? dz / sj * 0.5 : -yalf_dil + dz / sj * 0.5;
        double g12 = dxy / sj * 0.5, g23 = dyz / sj * 0.5, g31 = dzx / sj * 0.5;
        double hdd = g11 + g22 + g33;
        double fij = 2.0 * (f11 * g11 + f22 * g22 + f33 * g33) + f12 * g12 + f23 * g23 + f31 * g31;
        double cc7 = MC ? dlam * (fkk * hdd) + dmu * fij : dlam * (fkk * hdd) + dmu * fij + hdd;
        double dd_ = 1.0 / cc7;
        double df = dlam * fkk, dg = dlam * hdd;
        double ramda = (dmu2 * f11 - 3.0 * dlam * yalf) * de[0]
            + (dmu2 * f22 - 3.0 * dlam * yalf) * de[1]
            + (dmu2 * f33 - 3.0 * dlam * yalf) * de[2]
            + dmu * (f12 * de[3] + f23 * de[4] + f31 * de[5]);
        double ttt = ramda * dd_;
        if (ttt < 0.0) {
            double ww[6] = {dg + dmu2 * g11, dg + dmu2 * g22, dg + dmu2 * g33, dmu * g12, dmu * g23, dmu * g31};
            double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
            for (int a = 0; a < 6; a++)
                for (int b = 0; b < 6; b++) D[a][b] = D[a][b] - dd_ * ww[a] * zz[b];
            adps[0] = ramda * dd_ * f11; adps[1] = ramda * dd_ * f22; adps[2] = ramda * dd_ * f33;
            adps[3] = ramda * dd_ * f12; adps[4] = ramda * dd_ * f23; adps[5] = ramda * dd_ * f31;
        }
    }
}

// sub_camclay: subloading Cam-clay tangent (:129-281).  ymf from the
// critical-state ratio zmf; the subloading ratio term roue from log(sme0 / sm).
__device__ __forceinline__ void subcam_tangent(double D[6][6], double adps[6], const double s[6], const double de[6],
                                               double dlam, double dmu, double sm, double ann, double zmf,
                                               double zramda, double zkapa, double eps0, double sme0, double fs)
{
    const double dmu2 = dmu * 2.0;
    const double ymf = 3.0 * (zmf - 1.0) / (zmf + 2.0) / fs;
    const double hee = (zramda - zkapa) / (1.0 + eps0);
    double dx = -s[0] - sm, dy = -s[1] - sm, dz = -s[2] - sm;
    double dxy = -s[3], dyz = -s[4], dzx = -s[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double tt1 = 1.0 / (ymf * ymf * sm * sm + 3.0 * sjj);
    double tt2 = 2.0 * ymf * ymf * sm * tt1 - 1.0 / sm;
    double f11 = tt2 / 3.0 + dx * tt1 * 3.0;
    double f22 = tt2 / 3.0 + dy * tt1 * 3.0;
    double f33 = tt2 / 3.0 + dz * tt1 * 3.0;
    double f12 = 3.0 * dxy * tt1, f23 = 3.0 * dyz * tt1, f31 = 3.0 * dzx * tt1;
    double roue = (1 + eps0) * log(sme0 / sm);
    if (roue < 0.0) roue = 0.0;
    double ttt = ann * roue * roue;
    double hdd = f11 + f22 + f33 + ttt / sm;
    double fkk = f11 + f22 + f33;
    double fij = 2.0 * (f11 * f11 + f22 * f22 + f33 * f33) + f12 * f12 + f23 * f23 + f31 * f31;
    double cc7 = dlam * (fkk * fkk) + dmu * fij + hdd / hee;
    double dd_ = 1.0 / cc7;
    double df = dlam * fkk, dg = dlam * fkk;
    double ramda = (dmu2 * f11 + dlam * fkk) * de[0] + (dmu2 * f22 + dlam * fkk) * de[1]
        + (dmu2 * f33 + dlam * fkk) * de[2] + dmu * (f12 * de[3] + f23 * de[4] + f31 * de[5]);
    if (ramda < 0.0) {
        double ww[6] = {dg + dmu2 * f11, dg + dmu2 * f22, dg + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        for (int a = 0; a < 6; a++)
            for (int b = 0; b < 6; b++) D[a][b] = D[a][b] - dd_ * ww[a] * zz[b];
        adps[0] = ramda * dd_ * f11; adps[1] = ramda * dd_ * f22; adps[2] = ramda * dd_ * f33;
        adps[3] = ramda * dd_ * f12; adps[4] = ramda * dd_ * f23; adps[5] = ramda * dd_ * f31;
    }
}

// viscous_elastic (:88-126): dsig set directly, bulk modulus from the
// elastic modulus, shear modulus g = the material's c
__device__ __forceinline__ void visco_elastic(double ds[6], const double de[6], double e0, double poi, double g)
{
    const double k = e0 * 0.3333333333 / (1.0 - 2.0 * poi);
    const double epkk = de[0] + de[1] + de[2];
    ds[0] = 2.0 * g * (de[0] - epkk * 0.3333333333) + k * epkk;
    ds[1] = 2.0 * g * (de[1] - epkk * 0.3333333333) + k * epkk;
    ds[2] = 2.0 * g * (de[2] - epkk * 0.3333333333) + k * epkk;
    ds[3] = 2.0 * g * de[3];
    ds[4] = 2.0 * g * de[4];
    ds[5] = 2.0 * g * de[5];
}

// sub_camunsatu: unsaturated subloading Cam-clay (CPP_8-4-consfactor-umcc.cpp:
// 17-180).  D holds the elastic matrix of mean stress sm (taken with
// 0.333333333); the suction term follows the degree of saturation, and the
// plastic branch also sets the stress correction erfs.  ext points at the
// particle's SoilExt members (stride N).
static __device__ __noinline__ void unsat_tangent(double D[6][6], double adps[6], double erfs[6], const double s[6],
                                           const double de[6], double dlam, double dmu, double sm, double satu,
                                           double dsatu, double zmf, double fs, double zramda, double zkapa,
                                           double eps0, double sme0, double ann, double sitas, double sitar,
                                           const double* ext, int N)
{
    const double epss = ext[SX_EPSS * N], epsr = ext[SX_EPSR * N];
    const double bnn = ext[SX_BNN * N], beta = ext[SX_BETA * N];
    const double qq = (epsr - epss) / (sitas - sitar);
    const double dmu2 = dmu * 2.0;
    const double ymf = 3.0 * (zmf - 1.0) / (zmf + 2.0) / fs;
    const double hee = (zramda - zkapa) / (1.0 + eps0);
    const double dx = -s[0] - sm, dy = -s[1] - sm, dz = -s[2] - sm;
    const double dxy = -s[3], dyz = -s[4], dzx = -s[5];
    const double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    const double tt1 = 1.0 / (ymf * ymf * sm * sm + 3.0 * sjj);
    const double tt2 = 2.0 * ymf * ymf * sm * tt1 - 1.0 / sm;
    const double f11 = tt2 * 0.333333333 + dx * tt1 * 3.0;
    const double f22 = tt2 * 0.333333333 + dy * tt1 * 3.0;
    const double f33 = tt2 * 0.333333333 + dz * tt1 * 3.0;
    const double f12 = 3.0 * dxy * tt1, f23 = 3.0 * dyz * tt1, f31 = 3.0 * dzx * tt1;
    const double rous = qq * (sitas - satu);
    const double roue = hee * (1.0 + eps0) * log(sme0 / sm);
    double ttt = ann * roue + bnn * rous;
    ttt = pow(ttt, beta);
    const double hdd = f11 + f22 + f33 + ttt / sm;
    const double fkk = f11 + f22 + f33;
    const double fij = 2.0 * (f11 * f11 + f22 * f22 + f33 * f33) + f12 * f12 + f23 * f23 + f31 * f31;
    const double cc7 = dlam * (fkk * fkk) + dmu * fij + hdd / hee;
    const double dd_ = 1.0 / cc7;
    const double df = dlam * fkk, dg = dlam * fkk;
    double ramda = (dmu2 * f11 + dlam * fkk) * de[0] + (dmu2 * f22 + dlam * fkk) * de[1]
        + (dmu2 * f33 + dlam * fkk) * de[2] + dmu * (f12 * de[3] + f23 * de[4] + f31 * de[5]);
    const double omake = qq * dsatu / (zramda - zkapa);
    ramda = ramda + omake;
    if (ramda < 0.0) {
        erfs[0] = omake * dd_ * (D[0][0] * f11 + D[0][1] * f22 + D[0][2] * f33);
        erfs[1] = omake * dd_ * (D[1][0] * f11 + D[1][1] * f22 + D[1][2] * f33);
        erfs[2] = omake * dd_ * (D[2][0] * f11 + D[2][1] * f22 + D[2][2] * f33);
        erfs[3] = omake * dd_ * (D[3][3] * f12);
        erfs[4] = omake * dd_ * (D[4][4] * f23);
        erfs[5] = omake * dd_ * (D[5][5] * f31);
        const double ww[6] = {dg + dmu2 * f11, dg + dmu2 * f22, dg + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        const double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        for (int a = 0; a < 6; a++)
            for (int b = 0; b < 6; b++) D[a][b] = D[a][b] - dd_ * ww[a] * zz[b];
        adps[0] = ramda * dd_ * f11; adps[1] = ramda * dd_ * f22; adps[2] = ramda * dd_ * f33;
        adps[3] = ramda * dd_ * f12; adps[4] = ramda * dd_ * f23; adps[5] = ramda * dd_ * f31;
    }
}

// Minors of a 6x6 matrix for the cofactor expansion detA / getAStart use
// (CPP_8-5-consfactor-focc.cpp:265-322): the expansion of a k x k submatrix
// runs along its first row, over its columns in ascending order, and
// recurses into the remaining rows.  For a row list L (len 6, or 5 with one
// row left out) the submatrices met are the last k rows of L with a column
// set; each is evaluated once here, in ascending order of its column mask
// (a mask's subsets are smaller numbers), by the same operations the
// recursion applies to the same operands, so every value equals the
// recursive one.  M[mask] = det(rows L[len - popc(mask)..], columns of mask).
__device__ __forceinline__ void cofactor_minors(const double A[6][6], const int* L, int len, double M[64])
{
    for (int mask = 1; mask < 64; mask++) {
        const int k = __popc(mask);
        if (k > len) continue;
        const int r = L[len - k];
        if (k == 1) {
            M[mask] = A[r][__ffs(mask) - 1];
            continue;
        }
        double sum = 0;
        int t = 0;
        for (int col = 0; col < 6; col++) {
            if (!((mask >> col) & 1)) continue;
            sum += (t % 2 == 0 ? 1.0 : -1.0) * A[r][col] * M[mask & ~(1 << col)];
            t++;
        }
        M[mask] = sum;
    }
}

// dept = adjugate(T) / det(T) as fractional_mcc forms it (:223-246); a zero
// determinant takes the adjugate and determinant of C instead
static __device__ __noinline__ void adjugate_inverse(const double T[6][6], const double C[6][6], double D[6][6])
{
    const int all[6] = {0, 1, 2, 3, 4, 5};
    double M[64];
    const double (*A)[6] = T;
    cofactor_minors(A, all, 6, M);
    double det = M[63];
    if (det == 0.0) {
        A = C;
        cofactor_minors(A, all, 6, M);
        det = M[63];
    }
    for (int i = 0; i < 6; i++) {
        int L[5], q = 0;
        for (int r = 0; r < 6; r++)
            if (r != i) L[q++] = r;
        cofactor_minors(A, L, 5, M);
        for (int j = 0; j < 6; j++) {
            double adj = M[63 & ~(1 << j)];       // ans[j][i] of getAStart
            if ((i + j) % 2 == 1) adj = -adj;
            D[j][i] = adj / det;
        }
    }
}

// fractional_mcc: fractional-order plastic model of MCC (CPP_8-5-consfactor-focc.cpp:
// 13-247).  C is the elastic compliance, which fractional_plastic reuses; D the
// inverse of C (+ the plastic compliance n m / hp when the Cam-clay loading
// index is negative).  e is the particle's void ratio; pow(c, 4) comes
// precomputed.
static __device__ __noinline__ void focc_tangent(double D[6][6], double C[6][6], const double s[6], const double de[6],
                                          double e, double poi, double mc, double ramda, double alpha,
                                          const double* ext, int N)
{
    const double h1 = ext[SX_DAMP1 * N], h2 = ext[SX_DAMP2 * N], beta = ext[SX_BNN * N];
    const double zeta = ext[SX_ZET * N], etao = ext[SX_ETAO * N], g0 = ext[SX_G0 * N], c4 = ext[SX_C4 * N];
    const double p0 = 98000, pa = 98000;
    double sij[6], mij[6], nij[6], T[6][6];
    const double sm = (-s[0] + -s[1] + -s[2]) / 0.33333333;
    for (int a = 0; a < 6; a++) sij[a] = (a < 3) ? -s[a] - sm : -s[a];
    double q = 0.5 * (sij[0] * sij[0] + sij[1] * sij[1] + sij[2] * sij[2]) + sij[3] * sij[3] + sij[4] * sij[4] + sij[5] * sij[5];
    q = sqrt(3.0 * q);
    double ita = q / sm;
    if (ita == 0.0) {
        ita = 0.000001;
        q = ita * sm;
    }
    const double g = g0 * (2.97 - e) * (2.97 - e) / (1.0 + e) * sqrt(sm * pa);
    const double e0 = 2.0 * g * (1.0 + poi);
    const double ymf = mc;
    const double dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
    const double dmu = e0 * 0.5 / (1.0 + poi), dmu2 = dmu * 2.0;
    const double tt1 = 1.0 / (ymf * ymf * sm * sm + q * q);
    const double tt2 = 2.0 * ymf * ymf * sm * tt1 - 1.0 / sm;
    const double f11 = tt2 * 0.33333333 + sij[0] * tt1 * 3.0;
    const double f22 = tt2 * 0.33333333 + sij[1] * tt1 * 3.0;
    const double f33 = tt2 * 0.33333333 + sij[2] * tt1 * 3.0;
    const double f12 = 3.0 * sij[3] * tt1, f23 = 3.0 * sij[4] * tt1, f31 = 3.0 * sij[5] * tt1;
    const double fkk = f11 + f22 + f33;
    const double ramda_cc = (dmu2 * f11 + dlam * fkk) * de[0] + (dmu2 * f22 + dlam * fkk) * de[1]
        + (dmu2 * f33 + dlam * fkk) * de[2] + dmu * (f12 * de[3] + f23 * de[4] + f31 * de[5]);
    // Lode angle from the deviator's third and second invariants
    const double smn[3][3] = {{sij[0], sij[3], sij[5]}, {sij[3], sij[1], sij[4]}, {sij[5], sij[4], sij[2]}};
    double s_val = 0.0, skl = 0.0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int k = 0; k < 3; k++) s_val = s_val + smn[a][b] * smn[b][k] * smn[k][a];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) skl = skl + smn[a][b] * smn[b][a];
    if (skl == 0.0) skl = 0.000001;
    double sita = 9.0 * s_val * 0.5 / pow(1.5 * skl, 1.5);
    if (sita < -1.0) sita = -1.0;
    else if (sita > 1.0) sita = 1.0;
    sita = asin(sita) * 0.33333333;
    double m = 2 * c4 / (1 + c4 + (1 - c4) * sin(3.0 * sita));
    m = pow(m, 0.25);
    m = mc * m;
    const double pc = pa * pow((etao - e) / ramda, 1 / zeta);
    const double qc = q + m * (sm - pc);
    const double df = (sm - p0 / 2) * mc * mc / q;
    double dg = ((sm - pc) + (2 - alpha) * (pc - sm * 0.5 - q * q / mc / mc / sm / 2)) / ((q - qc) + (2 - alpha) * qc);
    dg = pow(m, alpha + 1) * dg;
    for (int a = 0; a < 6; a++) {
        mij[a] = 1.0 / sqrt(1.0 + df * df) * ((a < 3) ? 3.0 * sij[a] * 0.5 / q + df * 0.33333333 : 3.0 * sij[a] * 0.5 / q);
        nij[a] = 1.0 / sqrt(1.0 + dg * dg) * ((a < 3) ? 3.0 * sij[a] * 0.5 / q + dg * 0.33333333 : 3.0 * sij[a] * 0.5 / q);
    }
    const double order = beta * (e - etao + ramda * pow(sm / pa, zeta));
    const double mf = mc * pow(2.71828, -order);
    const double hp = (h1 - h2 * e) * (1 - e) * g * (mf - ita) / ita * pow(2.71828, order);
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) C[a][b] = 0.0;
    C[0][0] = 1.0 / e0; C[1][1] = 1.0 / e0; C[2][2] = 1.0 / e0;
    C[0][1] = -poi / e0; C[0][2] = -poi / e0; C[1][0] = -poi / e0;
    C[1][2] = -poi / e0; C[2][0] = -poi / e0; C[2][1] = -poi / e0;
    C[3][3] = 1.0 / g; C[4][4] = 1.0 / g; C[5][5] = 1.0 / g;
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) T[a][b] = (ramda_cc < 0.0) ? C[a][b] + nij[a] * mij[b] / hp : C[a][b];
    adjugate_inverse(T, C, D);
}

// fractional_plastic (:250-264): plastic strain rate = strain rate - C dsig
__device__ __forceinline__ void fractional_plastic(const double ds[6], const double de[6], double adps[6],
                                                   const double C[6][6])
{
    for (int a = 0; a < 6; a++) {
        double ee = 0.0;
        for (int b = 0; b < 6; b++) ee = ee + C[a][b] * ds[b];
        adps[a] = de[a] - ee;
    }
}

// TSSMP_before (CPP_7-3-TS.cpp:14-67): the transformed stress of the SMP
// criterion from the principal stresses sp of the last Stress_eigValue and
// the last deq's vsig / divq; s is replaced by it when q != 0.  Returns qc;
// ts receives the stress before the transformation.
__device__ __forceinline__ double tssmp_before(double s[6], double ts[6], const double sp[3], double vsig, double q,
                                               double alpha)
{
    double qc = 0.0, sx[6];
    sx[0] = -s[0] + vsig;
    sx[1] = -s[1] + vsig;
    sx[2] = -s[2] + vsig;
    sx[3] = -s[3]; sx[4] = -s[4]; sx[5] = -s[5];
    const double I1 = -(sp[0] + sp[1] + sp[2]);
    const double I2 = sp[0] * sp[1] + sp[1] * sp[2] + sp[2] * sp[1];
    const double I3 = -sp[0] * sp[1] * sp[2];
    if ((I1 * I1 - 3.0 * I2) >= 1.0e-7) {
        const double temp = 3.0 * sqrt((I1 * I2 - I3) / (I1 * I2 - 9.0 * I3)) - 1.0;
        if (fabs(temp) >= 1.0e-7)
            qc = alpha * sqrt(I1 * I1 - 3.0 * I2) + 2.0 * (1.0 - alpha) * I1 / (3.0 * sqrt((I1 * I2 - I3) / (I1 * I2 - 9.0 * I3)) - 1.0);
    }
    for (int a = 0; a < 6; a++) ts[a] = s[a];
    if (q != 0.0) {
        s[0] = -I1 * 0.33333333 - qc / q * sx[0];
        s[1] = -I1 * 0.33333333 - qc / q * sx[1];
        s[2] = -I1 * 0.33333333 - qc / q * sx[2];
        s[3] = -qc / q * sx[3];
        s[4] = -qc / q * sx[4];
        s[5] = -qc / q * sx[5];
    }
    return qc;
}

// TSSMP_after (:69-105): the stress rate back to the real stress space; s and
// ts exchange (s gets the stress before the transformation back)
__device__ __forceinline__ void tssmp_after(double ds[6], double s[6], double ts[6], double q, double qc)
{
    const double dvsig = (ds[0] + ds[1] + ds[2]) / 3.0;
    if (qc != 0.0) {
        ds[0] = dvsig + q / qc * (ds[0] - dvsig);
        ds[1] = dvsig + q / qc * (ds[1] - dvsig);
        ds[2] = dvsig + q / qc * (ds[2] - dvsig);
        ds[3] = q / qc * ds[3];
        ds[4] = q / qc * ds[4];
        ds[5] = q / qc * ds[5];
    }
    for (int a = 0; a < 6; a++) {
        const double t = ts[a];
        ts[a] = s[a];
        s[a] = t;
    }
}

// moisturesuct (CPP_7-2-constitutive.cpp:323-338): suction on the wetting
// (dsatu > 0) or drying curve, pi = 3.141592653 (Header_Parameters.h)
__device__ __forceinline__ double moisture_suction(double satu, double dsatu, double sitas, double sitar,
                                                   const double* ext, int N)
{
    const double temp = tan(3.141592653 * (sitas - satu) / (sitas - sitar) / 2.0);
    if (dsatu > 0.0) {
        const double c2 = ext[SX_C2 * N];
        return log(1 + exp(c2 * ext[SX_SW * N]) * temp) / c2;
    }
    const double c1 = ext[SX_C1 * N];
    return log(1 + exp(c1 * ext[SX_SD * N]) * temp) / c1;
}

// DPModel_check: stress-scaling return onto the cone (:779-819)
__device__ __forceinline__ void dp_check(const double s[6], double ds[6], double alpha_fai, double k_c, double dt)
{
    double ts[6];
    double sm = (s[0] + s[1] + s[2]) / 3.0;
    double dx = s[0] - sm, dy = s[1] - sm, dz = s[2] - sm;
    double sj_2 = 0.5 * (dx * dx + dy * dy + dz * dz) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    double sj = sqrt(sj_2);
    for (int a = 0; a < 6; a++) ts[a] = s[a] + ds[a] * dt;
    double i_1 = ts[0] + ts[1] + ts[2];
    double rn = (-alpha_fai * i_1 + k_c) / sj;
    if (rn < 1.0) {
        ts[0] = rn * (ts[0] - i_1 / 3.0) + i_1 / 3.0;
        ts[1] = rn * (ts[1] - i_1 / 3.0) + i_1 / 3.0;
        ts[2] = rn * (ts[2] - i_1 / 3.0) + i_1 / 3.0;
        ts[3] = rn * ts[3];
        ts[4] = rn * ts[4];
        ts[5] = rn * ts[5];
    }
    for (int a = 0; a < 6; a++) ds[a] = (ts[a] - s[a]) / dt;
}

// Particle::deq (Class_particle.cpp:121-143): vsig, veps, divq, divr
__device__ __forceinline__ void deq(const double s[6], const double ep[6], double* vsig, double* veps,
                                    double* divq, double* divr)
{
    *veps = ep[0] + ep[1] + ep[2];
    double vs = (s[0] + s[1] + s[2]) / 3;
    double sxx = s[0] - vs, syy = s[1] - vs, szz = s[2] - vs;
    double j2 = 0.5 * (sxx * sxx + syy * syy + szz * szz) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    double q = sqrt(3 * fabs(j2));
    *vsig = vs;
    *divq = q;
    *divr = (vs != 0.0) ? fabs(q / vs) : 0.0;
}

// Particle::shearstrain (Class_particle.cpp:175-192)
__device__ __forceinline__ double shearstrain(const double ep[6], double veps)
{
    double sxx = ep[0] - veps / 3.0, syy = ep[1] - veps / 3.0, szz = ep[2] - veps / 3.0;
    double j2 = 0.5 * (sxx * sxx + syy * syy + szz * szz) + ep[3] * ep[3] + ep[4] * ep[4] + ep[5] * ep[5];
    return sqrt(2.0 * fabs(j2));
}

// eejcb with its eigenvector matrix v (row-major, v[i*3+j]), as
// Stress_eigValue uses it for beta / beta_ts (CPP_7-1-strain.cpp:311-330,
// 341-437).
__device__ __forceinline__ void eig3v(const double s[6], double strep[3], double v[9])
{
    double a[9] = {s[0], s[3], s[5], s[3], s[1], s[4], s[5], s[4], s[2]};
    const int n = 3;
    for (int i = 0; i < 9; i++) v[i] = (i % 4 == 0) ? 1.0 : 0.0;
    int p = 0, q = 0, l = 1;
    while (true) {
        double fm = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double dd_ = fabs(a[i * n + j]);
                if ((i != j) && (dd_ > fm)) { fm = dd_; p = i; q = j; }
            }
        if (fm < 0.001) break;
        if (l > 7) break;
        l = l + 1;
        int u = p * n + q, w = p * n + p, t = q * n + p, sidx = q * n + q;
        double x = -a[u];
        double y = (a[sidx] - a[w]) / 2.0;
        double omega = x / sqrt(x * x + y * y);
        if (y < 0.0) omega = -omega;
        double sn = 1.0 + sqrt(1.0 - omega * omega);
        sn = omega / sqrt(2.0 * sn);
        double cn = sqrt(1.0 - sn * sn);
        fm = a[w];
        a[w] = fm * cn * cn + a[sidx] * sn * sn + a[u] * omega;
        a[sidx] = fm * sn * sn + a[sidx] * cn * cn - a[u] * omega;
        a[u] = 0.0;
        a[t] = 0.0;
        for (int j = 0; j < n; j++)
            if ((j != p) && (j != q)) {
                int uu = p * n + j, ww = q * n + j;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
        for (int i = 0; i < n; i++)
            if ((i != p) && (i != q)) {
                int uu = i * n + p, ww = i * n + q;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
        for (int i = 0; i < n; i++) {
            int uu = i * n + p, ww = i * n + q;
            fm = v[uu];
            v[uu] = fm * cn + v[ww] * sn;
            v[ww] = -fm * sn + v[ww] * cn;
        }
    }
    strep[0] = a[0]; strep[1] = a[4]; strep[2] = a[8];
}

// inverse_mat of the artificial stress (CPP_9-5-artificialstress.cpp:297-317):
// B is left unchanged (zero) when |det| <= 1e-5
__device__ __forceinline__ void inv3_or_keep(const double A[9], double B[9])
{
    const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[3] * (A[1] * A[8] - A[2] * A[7])
        + A[6] * (A[1] * A[5] - A[2] * A[4]);
    if (fabs(det) > 1.0e-5) {
        B[0] = (A[4] * A[8] - A[5] * A[7]) / det;
        B[1] = (A[2] * A[7] - A[1] * A[8]) / det;
        B[2] = (A[1] * A[5] - A[2] * A[4]) / det;
        B[3] = (A[5] * A[6] - A[3] * A[8]) / det;
        B[4] = (A[0] * A[8] - A[2] * A[6]) / det;
        B[5] = (A[3] * A[2] - A[0] * A[5]) / det;
        B[6] = (A[3] * A[7] - A[4] * A[6]) / det;
        B[7] = (A[1] * A[6] - A[0] * A[7]) / det;
        B[8] = (A[0] * A[4] - A[3] * A[1]) / det;
    }
}

// matrix_multiply (CPP_9-5-artificialstress.cpp:13-26), row-major 3x3
__device__ __forceinline__ void mul3(const double a[9], const double b[9], double c[9])
{
    for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) c[r * 3 + q] = a[r * 3] * b[q] + a[r * 3 + 1] * b[3 + q] + a[r * 3 + 2] * b[6 + q];
}

// eejcb Jacobi rotations, eps = 1e-3, at most 7 (CPP_7-1-strain.cpp:341-437);
// returns the diagonal (principal stresses strep).
__device__ __forceinline__ void eig3(const double s[6], double strep[3])
{
    double a[9] = {s[0], s[3], s[5], s[3], s[1], s[4], s[5], s[4], s[2]};
    const int n = 3;
    int p = 0, q = 0, l = 1;
    while (true) {
        double fm = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double dd_ = fabs(a[i * n + j]);
                if ((i != j) && (dd_ > fm)) { fm = dd_; p = i; q = j; }
            }
        if (fm < 0.001) break;
        if (l > 7) break;
        l = l + 1;
        int u = p * n + q, w = p * n + p, t = q * n + p, sidx = q * n + q;
        double x = -a[u];
        double y = (a[sidx] - a[w]) / 2.0;
        double omega = x / sqrt(x * x + y * y);
        if (y < 0.0) omega = -omega;
        double sn = 1.0 + sqrt(1.0 - omega * omega);
        sn = omega / sqrt(2.0 * sn);
        double cn = sqrt(1.0 - sn * sn);
        fm = a[w];
        a[w] = fm * cn * cn + a[sidx] * sn * sn + a[u] * omega;
        a[sidx] = fm * sn * sn + a[sidx] * cn * cn - a[u] * omega;
        a[u] = 0.0;
        a[t] = 0.0;
        for (int j = 0; j < n; j++)
            if ((j != p) && (j != q)) {
                int uu = p * n + j, ww = q * n + j;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
        for (int i = 0; i < n; i++)
            if ((i != p) && (i != q)) {
                int uu = i * n + p, ww = i * n + q;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
    }
    strep[0] = a[0]; strep[1] = a[4]; strep[2] = a[8];
}
