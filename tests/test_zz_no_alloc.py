"""The allocation-free dense inverse against the handle-based one.

skb_fft_inverse_device_noalloc is for callers that may not allocate device memory
while they run: a process that enforces its own device-memory budget through
its own allocator, or a plugin whose host forbids cudaMalloc / cudaFree inside
its compute callbacks (an allocation can fail once the budget is reserved, and
cudaFree stalls every stream on the device).  It needs no provider handle and
keeps its scratch in a fixed 64 MiB device array of the library.  These tests
check that two calls in a row, on different workloads and so with the array
rewritten in between, give what skb_fft_inverse_device gives for the same
spectrum, within the tolerances of the other GPU transform tests (1e-12
relative for FP64, 1e-5 for FP32), and that a workload needing more scratch
than the array holds is refused with a clear error.

This file is named to be collected last.
"""

import ctypes

import numpy as np
import pytest

import skb_cuda

pytestmark = pytest.mark.gpu

TOL = {skb_cuda.FP64: 1e-12, skb_cuda.FP32: 1e-5}
DTYPES = {skb_cuda.FP64: (np.float64, np.complex128), skb_cuda.FP32: (np.float32, np.complex64)}


def _noalloc(w, precision, spectrum_ptr, real_ptr, stream=None):
    lib = skb_cuda.library()
    skb_cuda.check(lib.skb_fft_inverse_device_noalloc(ctypes.byref(w), ctypes.c_int(precision),
                                                      ctypes.c_void_p(spectrum_ptr), ctypes.c_void_p(real_ptr),
                                                      ctypes.c_void_p(stream)))


def _case(w, precision, seed):
    real_t, complex_t = DTYPES[precision]
    rng = np.random.default_rng(seed)
    n = w.spectrum_elements
    spectrum = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(complex_t)
    d_spec = skb_cuda.DeviceArray.from_numpy(spectrum)
    d_real = skb_cuda.DeviceArray(w.real_elements * np.dtype(real_t).itemsize)
    provider = skb_cuda.FFTProvider(w, precision)
    provider.inverse_device(d_spec.ptr, d_real.ptr)
    skb_cuda.synchronize()
    expected = d_real.download(real_t, w.real_elements)
    provider.close()
    return d_spec, expected


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("precision", [skb_cuda.FP64, skb_cuda.FP32])
def test_two_calls_in_a_row_match_the_handle_inverse(precision):
    real_t, _ = DTYPES[precision]
    workloads = [skb_cuda.Workload(64, 32, 9, 2), skb_cuda.Workload(128, 128, 17, 3)]
    cases = [(w,) + _case(w, precision, 11 + i) for i, w in enumerate(workloads)]
    outs = [skb_cuda.DeviceArray(w.real_elements * np.dtype(real_t).itemsize) for w in workloads]
    # Two calls in a row on the default stream, then one synchronisation.
    for (w, d_spec, _), d_out in zip(cases, outs):
        _noalloc(w, precision, d_spec.ptr, d_out.ptr)
    skb_cuda.synchronize()
    for (w, _, expected), d_out in zip(cases, outs):
        got = d_out.download(real_t, w.real_elements)
        assert _rel_l2(got, expected) <= TOL[precision]
        assert np.max(np.abs(got - expected)) <= TOL[precision] * np.max(np.abs(expected))


def test_oversized_workload_is_refused():
    w = skb_cuda.Workload(1024, 1024, 65, 3)
    d = skb_cuda.DeviceArray(16)
    with pytest.raises(ValueError, match="bytes of scratch"):
        _noalloc(w, skb_cuda.FP64, d.ptr, d.ptr)


@pytest.mark.parametrize("precision", [skb_cuda.FP64, skb_cuda.FP32])
def test_matches_the_oracle_inverse(precision):
    # Against the CPU oracle's c2r (pocketfft in float64 with FFTW's
    # half-spectrum semantics), on a spectrum that is not Hermitian-consistent,
    # so the kx = 0 and Nyquist handling is exercised as well.
    from oracle import oracle as orc

    real_t, complex_t = DTYPES[precision]
    for shape, seed in (((64, 32, 9, 2), 31), ((256, 256, 5, 2), 32)):
        w = skb_cuda.Workload(*shape)
        rng = np.random.default_rng(seed)
        n = w.spectrum_elements
        spectrum = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(complex_t)
        d_spec = skb_cuda.DeviceArray.from_numpy(spectrum)
        d_real = skb_cuda.DeviceArray(w.real_elements * np.dtype(real_t).itemsize)
        _noalloc(w, precision, d_spec.ptr, d_real.ptr)
        skb_cuda.synchronize()
        got = d_real.download(real_t, w.real_elements)
        ref = orc.fft_c2r(orc.Workload(*shape), spectrum.astype(np.complex128))
        assert orc.rel_l2_error(got, ref) <= TOL[precision]
        assert orc.max_rel_error(got, ref) <= TOL[precision]
