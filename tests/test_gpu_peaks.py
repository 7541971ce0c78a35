"""The measured FP64 / FP32 multiply-add rates (sphgpu_pipe_peaks), the
compute denominators of bench.py's FP64 roofline."""
import pytest

import sphgpu

pytestmark = pytest.mark.gpu


def test_pipe_peaks_are_plausible():
    f64, f32 = sphgpu.pipe_peaks(0)
    print("FP64 %.1f TFLOP/s, FP32 %.1f TFLOP/s" % (f64, f32))
    # a B200 runs tens of TFLOP/s in either; FP32 is not slower than FP64
    assert 1.0 < f64 < 1000.0
    assert 1.0 < f32 < 1000.0
    assert f32 >= 0.9 * f64


def test_pipe_peaks_bad_device():
    with pytest.raises(sphgpu.SPHError):
        sphgpu.pipe_peaks(999)
