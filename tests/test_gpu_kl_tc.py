"""Batched K-L synthesis on the tensor cores (sphgpu_kl_synthesize) against
the FP64 generator (sphgpu_kl_generate, itself within 2e-15 of the
reference's own output).

R realisations share the geometry; the K-term sum runs as tcgen05 TF32 MMAs
on split operands (three products), accumulating in FP32 in tensor memory.
Each realisation is held to TC_REL_TOL of the FP64 field, relative to the
field's largest magnitude; NaN marks particles a field does not cover, in
both.
"""
import numpy as np
import pytest

import scenes
import sphgpu

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TC_REL_TOL = 2e-5


def _setup(sc):
    st = scenes.initialise(sc)
    eng = sphgpu.Engine(st.params, device=0)
    eng.load_state(st.fields, st.fluid, st.soil)
    dom = scenes.kl_domain(sc)
    return eng, sphgpu.kl_domain(dom["nb_min"], dom["nb_max"], dom["soil_max"], dom["water_max"])


@pytest.mark.parametrize("label,factory,field,R", [
    ("slope_2d_cohesion", lambda: scenes.slope_2d(H=5.0, dx=0.1),
     sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [10.0, 1.0]), 32),
    ("column_3d_friction", lambda: scenes.soil_column_3d(dx=0.05, steps=100),
     sphgpu.kl_field(0, 1, 30.0, 3.0, [0.5, 0.3, 0.2], 2.0), 48),
    ("column_3d_fluid_lognormal_R256", lambda: scenes.soil_column_3d(dx=0.05, steps=100),
     sphgpu.kl_field(5, 2, 50.0, 10.0, [0.4, 0.4, 0.3]), 256),
])
def test_synthesis_matches_fp64_generator(label, factory, field, R):
    sc = factory()
    eng, dom = _setup(sc)
    K = 200
    xi = np.random.default_rng(R).standard_normal((R, K))
    out = torch.full((R * eng.n,), float("nan"), dtype=torch.float32, device="cuda")
    ms = eng.kl_synthesize(dom, field, xi, out.data_ptr(), K)
    got = out.cpu().numpy().reshape(R, eng.n).astype(np.float64)
    worst = 0.0
    for r in list(range(0, R, max(1, R // 8)))[:8] + [R - 1]:
        ref = eng.kl_generate(dom, [field], xi[r][None, :], K)[0]
        assert np.array_equal(np.isnan(got[r]), np.isnan(ref)), r
        m = ~np.isnan(ref)
        err = float(np.abs(got[r][m] - ref[m]).max() / np.abs(ref[m]).max())
        worst = max(worst, err)
        assert err <= TC_REL_TOL, (r, err)
    print(f"{label}: R={R} K={K} n={eng.n} kernel {ms:.3f} ms, worst relative error {worst:.2e}")


def test_synthesis_rejects_bad_shapes():
    eng, dom = _setup(scenes.slope_2d(H=5.0, dx=0.1))
    out = torch.empty(24 * eng.n, dtype=torch.float32, device="cuda")
    with pytest.raises(sphgpu.SPHError) as e:
        eng.kl_synthesize(dom, sphgpu.kl_field(1, 1, 1.0, 0.1, [1.0, 1.0]), np.zeros((24, 200)), out.data_ptr())
    assert e.value.code == 100


def test_bounded_wait_expires_and_context_stays_usable():
    """The synthesis kernel's bounded completion wait, made to run out on a
    barrier that nothing signals (sphgpu_kl_wait_check, about 0.5 ms of SM
    clock): the call reports SPHGPU_E_KL_TIMEOUT (105), and the next synthesis
    on the same context, which needs the tensor memory the timed-out CTA held,
    runs and is correct."""
    sc = scenes.slope_2d(H=5.0, dx=0.1)
    eng, dom = _setup(sc)
    for _ in range(2):
        assert eng.lib.sphgpu_kl_wait_check(eng.h, 1_000_000) == 105
    field = sphgpu.kl_field(1, 2, 10.0e3, 3.0e3, [10.0, 1.0])
    R, K = 16, 200
    xi = np.random.default_rng(5).standard_normal((R, K))
    out = torch.full((R * eng.n,), float("nan"), dtype=torch.float32, device="cuda")
    eng.kl_synthesize(dom, field, xi, out.data_ptr(), K)
    got = out.cpu().numpy().reshape(R, eng.n).astype(np.float64)
    ref = eng.kl_generate(dom, [field], xi[3][None, :], K)[0]
    m = ~np.isnan(ref)
    assert float(np.abs(got[3][m] - ref[m]).max() / np.abs(ref[m]).max()) <= TC_REL_TOL
