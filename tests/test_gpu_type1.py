"""GPU parity of the constant-stratification type-I vertical transforms
(DCT-I = FFTW REDFT00, DST-I = RODFT00 on the interior, WVM forward
normalisation, the production call schedule) against the oracle, which is
pinned to scipy's pocketfft type-I transforms in test_oracle_pins.py.

Tolerances: FP64 1e-12 (the reference's constant-stratification tolerance,
src/constant_stratification.cpp:30), FP32 1e-5 relative L2 against the oracle
on the FP32-rounded input.  Channels outside the transformed range, and the
DST endpoints of a raw DST, must come back bit-identical."""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

KINDS = {"dct": skb_cuda.TYPE1_DCT, "dst": skb_cuda.TYPE1_DST}


def _data(rows, storage, nz, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((rows, storage, nz)) + 1j * rng.standard_normal((rows, storage, nz))


def _round32(x):
    return x.real.astype(np.float32).astype(np.float64) + 1j * x.imag.astype(np.float32).astype(np.float64)


# nz = 3, 7, 130: direct sums; the others: warp FFT of the 2(nz-1) extension.
@pytest.mark.parametrize("nz", [3, 7, 9, 33, 65, 129, 130, 257, 513])
@pytest.mark.parametrize("kind", ["dct", "dst"])
@pytest.mark.parametrize("normalize", [False, True])
def test_fp64_against_oracle(nz, kind, normalize):
    rows, storage, first, channels = 37, 3, 1, 2
    x = _data(rows, storage, nz, 100 + nz)
    t = skb_cuda.ConstantStratificationVertical(rows, nz, skb_cuda.FP64)
    got = t.transform(x, KINDS[kind], storage, first, channels, normalize).reshape(rows, storage, nz)
    want = orc.type1_transform(x, kind, storage, first, channels, normalize)
    sel = slice(first, first + channels)
    assert orc.max_rel_error(got[:, sel], want[:, sel]) <= 1e-12
    assert orc.rel_l2_error(got[:, sel], want[:, sel]) <= 1e-12
    # Untouched channel 0 and, for a raw DST, untouched endpoints.
    assert np.array_equal(got[:, 0], x[:, 0])
    if kind == "dst" and not normalize:
        assert np.array_equal(got[:, sel, 0], x[:, sel, 0])
        assert np.array_equal(got[:, sel, nz - 1], x[:, sel, nz - 1])
    if kind == "dst" and normalize:
        assert not np.any(got[:, sel, 0]) and not np.any(got[:, sel, nz - 1])


@pytest.mark.parametrize("nz", [9, 65, 129, 130])
@pytest.mark.parametrize("kind", ["dct", "dst"])
def test_fp32_against_oracle(nz, kind):
    rows, storage = 41, 1
    x = _data(rows, storage, nz, 7 * nz)
    t = skb_cuda.ConstantStratificationVertical(rows, nz, skb_cuda.FP32)
    got = t.transform(x, KINDS[kind], storage, 0, 1, True).reshape(rows, storage, nz)
    want = orc.type1_transform(_round32(x), kind, storage, 0, 1, True)
    assert orc.rel_l2_error(got, want) <= 1e-5


def test_device_form_and_normalisation_pass():
    rows, storage, nz = 53, 3, 65
    x = _data(rows, storage, nz, 5)
    t = skb_cuda.ConstantStratificationVertical(rows, nz, skb_cuda.FP64)
    d = skb_cuda.DeviceArray.from_numpy(x.reshape(-1))
    t.transform_device(d.ptr, skb_cuda.TYPE1_DCT, storage, 0, 2)
    t.normalize_device(d.ptr, skb_cuda.TYPE1_DCT, storage, 0, 2)
    t.transform_device(d.ptr, skb_cuda.TYPE1_DST, storage, 2, 1, normalize=True)
    skb_cuda.synchronize()
    got = d.download(np.complex128, x.size).reshape(rows, storage, nz)
    want = orc.type1_transform(orc.type1_transform(x, "dct", storage, 0, 2, True), "dst", storage, 2, 1, True)
    assert orc.max_rel_error(got, want) <= 1e-12
    # The separate normalisation pass equals the fused one.
    fused = t.transform(x, skb_cuda.TYPE1_DCT, storage, 0, 2, True).reshape(rows, storage, nz)
    assert orc.max_rel_error(got[:, :2], fused[:, :2]) <= 1e-15


@pytest.mark.parametrize("n,nz", [(8, 7), (32, 33), (64, 65)])
def test_schedule_compact_matches_full_half_and_oracle(n, nz):
    """The reference's schedule check (constant_stratification.cpp:541-557):
    the production call graph on the retained compact rows equals it on the
    full half-spectrum rows at the same (stored kx, ky), conjugated where the
    mode stores its conjugate; and both equal the oracle's schedule."""
    nx_half = n // 2 + 1
    full_rows = n * nx_half
    modes = orc.retained_modes(n, n)
    ids = modes.kx + nx_half * modes.ky
    full3 = orc.type1_deterministic(full_rows, 3, nz)
    full1 = orc.type1_deterministic(full_rows, 1, nz)
    comp3 = orc.type1_deterministic(len(modes), 3, nz, ids, modes.conj)
    comp1 = orc.type1_deterministic(len(modes), 1, nz, ids, modes.conj)
    f3, f1 = skb_cuda.ConstantStratificationVertical(full_rows, nz).schedule(full3, full1)
    c3, c1 = skb_cuda.ConstantStratificationVertical(len(modes), nz).schedule(comp3, comp1)
    f3 = f3.reshape(full_rows, 3, nz)
    f1 = f1.reshape(full_rows, 1, nz)
    c3 = c3.reshape(-1, 3, nz)
    c1 = c1.reshape(-1, 1, nz)
    ref3 = np.where(modes.conj[:, None, None], np.conj(f3[ids]), f3[ids])
    ref1 = np.where(modes.conj[:, None, None], np.conj(f1[ids]), f1[ids])
    assert orc.max_rel_error(c3, ref3) <= 1e-12 and orc.rel_l2_error(c3, ref3) <= 1e-12
    assert orc.max_rel_error(c1, ref1) <= 1e-12 and orc.rel_l2_error(c1, ref1) <= 1e-12
    o3, o1 = orc.type1_schedule(full3, full1)
    assert orc.rel_l2_error(f3, o3) <= 1e-12 and orc.rel_l2_error(f1, o1) <= 1e-12


def test_schedule_device_matches_host():
    rows, nz = 97, 129
    a3 = _data(rows, 3, nz, 11)
    a1 = _data(rows, 1, nz, 12)
    t = skb_cuda.ConstantStratificationVertical(rows, nz, skb_cuda.FP64)
    h3, h1 = t.schedule(a3, a1)
    d3 = skb_cuda.DeviceArray.from_numpy(a3.reshape(-1))
    d1 = skb_cuda.DeviceArray.from_numpy(a1.reshape(-1))
    t.schedule_device(d3.ptr, d1.ptr)
    skb_cuda.synchronize()
    assert np.array_equal(d3.download(np.complex128, a3.size), h3.reshape(-1))
    assert np.array_equal(d1.download(np.complex128, a1.size), h1.reshape(-1))


def test_invalid_arguments_are_refused():
    with pytest.raises(ValueError):
        skb_cuda.ConstantStratificationVertical(4, 2)
    t = skb_cuda.ConstantStratificationVertical(4, 9)
    x = _data(4, 3, 9, 1)
    with pytest.raises(ValueError):
        t.transform(x, 7, 3, 0, 1)
    with pytest.raises(ValueError):
        t.transform(x, skb_cuda.TYPE1_DCT, 3, 2, 2)
