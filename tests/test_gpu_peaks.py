"""Measured SIMT FMA peaks (the compute side of the row kernel's roofline)."""

import pytest

import skb_cuda

pytestmark = pytest.mark.gpu


def test_simt_peaks_are_measured_and_plausible():
    f32, f64 = skb_cuda.simt_peaks()
    # A B200 runs FP32 FMAs at tens of TFLOP/s and FP64 at a fraction of that;
    # the bounds only catch a broken measurement, not a slow GPU.
    assert 5.0 < f32 < 300.0, f32
    assert 0.5 < f64 < f32, (f32, f64)
