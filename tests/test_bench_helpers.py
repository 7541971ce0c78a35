"""bench.py's roofline arithmetic on the CPU: the per-pass algorithmic bytes
(the compulsory traffic of a barrier-level pass list, 806 B per particle and
step for the 2-D dam break, 1,870 B for the 3-D soil column), the mapping of
stage times onto passes, and the FP64 roofline's failure path."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_pass_bytes_sum_to_the_step_figures():
    assert sum(bench.pass_bytes(2).values()) == pytest.approx(806.0)
    assert sum(bench.pass_bytes(3).values()) == pytest.approx(bench.STEP_BYTES_3D)
    assert set(bench.PASS_KERNELS) == set(bench.PASS_BYTES_2D)


def test_pass_roofline_from_stage_times():
    n = 1_000_000
    stages = {"k_density": 2.0, "k_shepard_eos": 1.0, "k_accel_a": 1.5, "k_accel_b": 3.5, "reorder": 0.0}
    out = bench.pass_roofline(stages, n, 6650.0)
    mom = out["stress divergence + viscosity + walls + velocity update"]
    assert mom["ms"] == pytest.approx(5.0)
    want = mom["bytes_per_particle"] * n / 5.0e-3 / 1e9
    assert mom["achieved_gbs"] == pytest.approx(want)
    assert mom["frac"] == pytest.approx(want / 6650.0)
    # a pass whose kernels did not run reports no rate
    assert out["reorder"]["ms"] == 0.0 and out["reorder"]["achieved_gbs"] is None
    assert out["key"]["frac"] is None


def test_fp64_roofline_reports_an_unavailable_measurement(monkeypatch):
    sys.path.insert(0, bench.PKG)
    import sphgpu

    def fail(device=0):
        raise sphgpu.SPHError(102, "sphgpu_pipe_peaks")
    monkeypatch.setattr(sphgpu, "pipe_peaks", fail)
    out = bench.fp64_roofline(0, 1000, 10.0)
    assert "unavailable" in out


def test_fp64_roofline_arithmetic(monkeypatch):
    sys.path.insert(0, bench.PKG)
    import sphgpu
    monkeypatch.setattr(sphgpu, "pipe_peaks", lambda device=0: (40.0, 80.0))
    out = bench.fp64_roofline(0, 2_000_000, 20.0)
    want = bench.STEP_FLOPS_3D * 2_000_000 / 0.020 / 1e12
    assert out["achieved"] == pytest.approx(want)
    assert out["frac"] == pytest.approx(want / 40.0)
    assert out["fp32_peak"] == 80.0
