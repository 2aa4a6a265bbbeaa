"""GPU parity of the WVM-direct vertical GEMM provider (vertical_gemm.cpp:935-1169):
per-mode grouped GEMM on full WVM-order spectra with the kx = 0 boundary copy,
against the oracle's restatement, at the FP64 1e-12 tolerance and the split
TF32x3 / FP32 tolerances (1e-6 / 1e-5 relative L2)."""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

TOL = {skb_cuda.GEMM_FP64: 1e-12, skb_cuda.GEMM_TF32X3: 1e-6, skb_cuda.GEMM_FP32: 1e-5}


def setup(nx, nz, fields, precision):
    w = skb_cuda.Workload(nx, nx, nz, fields)
    ow = orc.Workload(nx, nx, nz, fields)
    fam = orc.k2_family(ow)
    groups = skb_cuda.squared_wavenumber_groups(w)
    p = skb_cuda.WvmDirectVerticalProvider(w, groups, fam[0].reshape(-1), fam[1].reshape(-1),
                                           gemm_precision=precision)
    return w, ow, fam, p


def rand(rng, n):
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


@pytest.mark.parametrize("shape", [(16, 9, 3), (64, 17, 2)])
@pytest.mark.parametrize("precision", [skb_cuda.GEMM_FP64, skb_cuda.GEMM_TF32X3, skb_cuda.GEMM_FP32])
def test_host_forms_match_oracle(shape, precision):
    w, ow, fam, p = setup(*shape, precision)
    rng = np.random.default_rng(sum(shape) + precision)
    spec = rand(rng, p.spectrum_elements)
    modal = rand(rng, p.modal_elements)
    got_f = p.forward(spec)
    want_f = orc.wvm_direct_vertical(ow, fam, "forward", spec)
    got_i = p.inverse(modal)
    want_i = orc.wvm_direct_vertical(ow, fam, "inverse", modal)
    if precision == skb_cuda.GEMM_FP64:
        assert orc.max_rel_error(got_f, want_f) <= TOL[precision]
        assert orc.max_rel_error(got_i, want_i) <= TOL[precision]
    assert orc.rel_l2_error(got_f, want_f) <= TOL[precision]
    assert orc.rel_l2_error(got_i, want_i) <= TOL[precision]


def test_untouched_cells_keep_caller_values_and_partners_are_conjugate():
    w, ow, fam, p = setup(16, 9, 3, skb_cuda.GEMM_FP64)
    rng = np.random.default_rng(5)
    spec = rand(rng, p.spectrum_elements)
    prior = rand(rng, p.modal_elements)
    got = p.forward(spec, out=prior)
    want = orc.wvm_direct_vertical(ow, fam, "forward", spec, out=prior)
    assert orc.max_rel_error(got, want) <= 1e-12
    half = w.nx_half
    y = got.reshape(w.ny, half, w.fields, w.nj)
    modes = orc.retained_modes(16, 16)
    for kx, ky in zip(modes.kx, modes.ky):
        if kx == 0 and ky != 0 and 2 * ky != w.ny:
            assert np.array_equal(y[(w.ny - ky) % w.ny, 0], np.conj(y[ky, 0]))
    retained = np.zeros((w.ny, half), bool)
    retained[modes.ky, modes.kx] = True
    for kx, ky in zip(modes.kx, modes.ky):
        if kx == 0 and ky != 0:
            retained[(w.ny - ky) % w.ny, 0] = True
    assert np.array_equal(y[~retained], prior.reshape(w.ny, half, w.fields, w.nj)[~retained])


def test_device_forms_match_host_forms():
    w, ow, fam, p = setup(64, 17, 2, skb_cuda.GEMM_FP64)
    rng = np.random.default_rng(9)
    spec = rand(rng, p.spectrum_elements)
    d_spec = skb_cuda.DeviceArray.from_numpy(spec)
    d_modal = skb_cuda.DeviceArray.from_numpy(np.zeros(p.modal_elements, np.complex128))
    p.forward_device(d_spec.ptr, d_modal.ptr)
    skb_cuda.synchronize()
    got = d_modal.download(np.complex128, p.modal_elements)
    assert np.array_equal(got, p.forward(spec))
    d_back = skb_cuda.DeviceArray.from_numpy(np.zeros(p.spectrum_elements, np.complex128))
    p.inverse_device(d_modal.ptr, d_back.ptr)
    skb_cuda.synchronize()
    assert np.array_equal(d_back.download(np.complex128, p.spectrum_elements), p.inverse(got))
