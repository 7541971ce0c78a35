"""sphgpu_nnps_noalloc: the neighbour search for callers that cannot allocate
device memory (memory pools that forbid new allocations, real-time loops,
hosts that own every device buffer).  It keeps its intermediates in one fixed
array inside the library, so the test allocates the input and output buffers
itself (with torch) and hands their device pointers over.

The lists must equal those of the context-based search (sphgpu_nnps) on the
same positions, on two calls in a row (the second call reuses the array the
first one left behind).  Neighbour lists are integers: the comparison is
exact.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import scenes
import sphgpu

pytestmark = pytest.mark.gpu


def _case(scene):
    import torch
    st = scenes.initialise(scene)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    n = eng.n
    dev = torch.device("cuda", 0)
    xp = torch.tensor(np.ascontiguousarray(st.fields["xp"]), dtype=torch.float64, device=dev)
    hl = torch.tensor(np.ascontiguousarray(st.fields["hl"]), dtype=torch.float64, device=dev)
    ty = torch.tensor(np.ascontiguousarray(st.fields["type"]), dtype=torch.int32, device=dev)
    return eng, n, xp, hl, ty


@pytest.mark.parametrize("factory", [
    lambda: scenes.dam_break_2d(dx=0.01, steps=10),
    lambda: scenes.soil_column_3d(dx=0.05, steps=10),
])
def test_noalloc_nnps_matches_context_search(factory):
    import torch
    eng, n, xp, hl, ty = _case(factory())
    assert n <= 65536
    lib = sphgpu.load_library()
    lib.sphgpu_nnps_noalloc.argtypes = [C.POINTER(sphgpu.Params), C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.sphgpu_nnps_noalloc_scratch_bytes.restype = C.c_size_t
    assert 0 < lib.sphgpu_nnps_noalloc_scratch_bytes() < (64 << 20)
    want_n, want_l = eng.nnps()
    for call in range(2):
        ninflu = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        influ = torch.zeros((n, 100), dtype=torch.int32, device="cuda")
        rc = lib.sphgpu_nnps_noalloc(C.byref(eng.params), n, C.c_void_p(xp.data_ptr()),
                                     C.c_void_p(hl.data_ptr()), C.c_void_p(ty.data_ptr()),
                                     C.c_void_p(ninflu.data_ptr()), C.c_void_p(influ.data_ptr()), None)
        assert rc == 0, (call, rc)
        got_n = ninflu.cpu().numpy()
        got_l = influ.cpu().numpy()
        assert np.array_equal(got_n, want_n), call
        mask = np.arange(100)[None, :] <= np.minimum(want_n, 99)[:, None]
        mask[:, 0] = False
        assert np.array_equal(np.where(mask, got_l, 0), np.where(mask, want_l, 0)), call
    eng.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = sphgpu.load_library()
    lib.sphgpu_nnps_noalloc.argtypes = [C.POINTER(sphgpu.Params), C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    st = scenes.initialise(scenes.dam_break_2d(dx=0.02, steps=10))
    p = sphgpu.params_from_dict(st.params)
    dummy = C.c_void_p(16)   # never dereferenced: the size check comes first
    rc = lib.sphgpu_nnps_noalloc(C.byref(p), 65536 + 1, dummy, dummy, dummy, dummy, dummy, None)
    assert rc == 100


def _lib():
    lib = sphgpu.load_library()
    lib.sphgpu_nnps_noalloc.argtypes = [C.POINTER(sphgpu.Params), C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def _call(lib, params, n, xp, hl, ty, ninflu, influ, stream=None):
    return lib.sphgpu_nnps_noalloc(C.byref(params), n, C.c_void_p(xp.data_ptr()), C.c_void_p(hl.data_ptr()),
                                   C.c_void_p(ty.data_ptr()), C.c_void_p(ninflu.data_ptr()),
                                   C.c_void_p(influ.data_ptr()), stream)


def test_noalloc_rejects_grids_beyond_its_scratch():
    """A grid of more cells than the fixed array holds is refused before any
    pointer is read."""
    lib = _lib()
    st = scenes.initialise(scenes.dam_break_2d(dx=0.02, steps=10))
    p = sphgpu.params_from_dict(st.params)
    p.cxm, p.cym, p.czm = 1024, 257, 1
    p.ctotal = p.cxm * p.cym
    assert p.ctotal > 262144
    dummy = C.c_void_p(16)
    assert lib.sphgpu_nnps_noalloc(C.byref(p), 100, dummy, dummy, dummy, dummy, dummy, None) == 100


def test_noalloc_particle_outside_grid_returns_3_and_writes_nothing():
    """A particle beyond the cell grid: code 3 (parttocell), and neither the
    counts nor the lists are written."""
    import torch
    eng, n, xp, hl, ty = _case(scenes.dam_break_2d(dx=0.02, steps=10))
    xp[5, 0] = float(eng.params.xmax) + 50.0 * float(eng.params.dr)
    ninflu = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    influ = torch.full((n, 100), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert _call(_lib(), eng.params, n, xp, hl, ty, ninflu, influ) == 3
    assert (ninflu.cpu().numpy() == -1).all()
    assert (influ.cpu().numpy() == -7).all()
    eng.close()


def test_noalloc_too_many_neighbours_returns_5_with_every_count():
    """150 water particles packed into a 1 cm patch have more than 99
    neighbours: code 5 (partisearching), with every count written and no
    list slot beyond 99."""
    import torch
    sc = scenes.dam_break_2d(dx=0.02, steps=10)
    water = np.flatnonzero(sc.ptype == 1)[:150]
    sc.xp[water, 0] = 0.2 + 0.001 * (np.arange(150) % 10)
    sc.xp[water, 1] = 0.2 + 0.001 * (np.arange(150) // 10)
    eng, n, xp, hl, ty = _case(sc)
    ninflu = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    influ = torch.zeros((n, 100), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert _call(_lib(), eng.params, n, xp, hl, ty, ninflu, influ) == 5
    got = ninflu.cpu().numpy()
    assert (got >= 0).all()
    assert got[water].max() > 99
    eng.close()


def test_noalloc_on_a_caller_stream():
    """The search on a non-default stream the caller owns gives the same
    lists as the context-based search."""
    import torch
    eng, n, xp, hl, ty = _case(scenes.dam_break_2d(dx=0.01, steps=10))
    want_n, want_l = eng.nnps()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        ninflu = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        influ = torch.zeros((n, 100), dtype=torch.int32, device="cuda")
    rc = _call(_lib(), eng.params, n, xp, hl, ty, ninflu, influ, C.c_void_p(s.cuda_stream))
    assert rc == 0
    s.synchronize()
    got_n, got_l = ninflu.cpu().numpy(), influ.cpu().numpy()
    assert np.array_equal(got_n, want_n)
    mask = np.arange(100)[None, :] <= np.minimum(want_n, 99)[:, None]
    mask[:, 0] = False
    assert np.array_equal(np.where(mask, got_l, 0), np.where(mask, want_l, 0))
    eng.close()
