"""GPU parity of the horizontal transforms (full 2-D r2c/c2r and pruned)
against the reference's golden vectors and the pinned CPU oracle.

Tolerances: FP64 paths 1e-12 relative (max-relative and relative-L2, the
reference's own tolerance, benchmark.cpp:47); FP32 paths 1e-5 relative-L2.
"""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-12


def ow(w):
    return orc.Workload(w.nx, w.ny, w.nz, w.fields)


def test_fft_smoke_fixtures_match_direct_dft(golden_vectors):
    # validate --profile smoke (benchmark.cpp:4921-4936).
    g = golden_vectors
    w = skb_cuda.Workload(8, 8, 7, 2)
    fft = skb_cuda.FFTProvider(w)
    for i in range(5):
        real = g[f"smoke_{i}_real"]
        spec = fft.forward(real)
        assert orc.max_rel_error(spec, g[f"smoke_{i}_spectrum"]) <= TOL
        assert orc.rel_l2_error(spec, g[f"smoke_{i}_spectrum"]) <= TOL
        back = fft.inverse(g[f"smoke_{i}_spectrum"])
        assert orc.max_rel_error(back, g[f"smoke_{i}_c2r"]) <= TOL
        # inverse normalisation: c2r(r2c(x)) / (Nx*Ny) == x
        assert orc.max_rel_error(fft.inverse(spec) / 64.0, real) <= TOL


def test_fft_direct_dft_32(golden_vectors):
    g = golden_vectors
    w = skb_cuda.Workload(32, 32, 3, 2)
    fft = skb_cuda.FFTProvider(w)
    spec = fft.forward(g["d32_real"])
    assert orc.max_rel_error(spec, g["d32_spectrum"]) <= TOL
    assert orc.rel_l2_error(spec, g["d32_spectrum"]) <= TOL
    assert orc.max_rel_error(fft.inverse(g["d32_spectrum"]), g["d32_c2r"]) <= TOL


def test_fft_quick_profile_random_matches_oracle():
    # 195 planes of 256x256 (3 fields x Nz=65), makeFixture(random, 129).
    w = skb_cuda.Workload(256, 256, 65, 3)
    real = skb_cuda.make_fixture(w, "random", 129)
    fft = skb_cuda.FFTProvider(w)
    spec = fft.forward(real)
    expected = orc.fft_r2c(ow(w), real)
    assert orc.max_rel_error(spec, expected) <= TOL
    assert orc.rel_l2_error(spec, expected) <= TOL
    back = fft.inverse(spec)
    assert orc.max_rel_error(back / (256 * 256), real) <= TOL
    assert orc.max_rel_error(back, orc.fft_c2r(ow(w), spec)) <= TOL


@pytest.mark.parametrize("nx,ny,nz,f", [(4, 8, 3, 1), (8, 4, 2, 2), (2, 16, 3, 1), (16, 2, 2, 1), (64, 128, 5, 2),
                                        (128, 32, 9, 1), (1024, 8, 2, 1), (8, 1024, 2, 1), (512, 512, 3, 1)])
def test_fft_shapes_match_oracle(nx, ny, nz, f):
    w = skb_cuda.Workload(nx, ny, nz, f)
    real = skb_cuda.make_fixture(w, "random", 700)
    fft = skb_cuda.FFTProvider(w)
    spec = fft.forward(real)
    assert orc.rel_l2_error(spec, orc.fft_r2c(ow(w), real)) <= TOL
    # FFTW c2r semantics on a non-Hermitian spectrum (imaginary DC / Nyquist ignored).
    rng = np.random.default_rng(3)
    arb = rng.standard_normal(w.spectrum_elements) + 1j * rng.standard_normal(w.spectrum_elements)
    assert orc.max_rel_error(fft.inverse(arb), orc.fft_c2r(ow(w), arb)) <= TOL


def test_fft_inverse_preserves_input():
    w = skb_cuda.Workload(32, 32, 3, 1)
    fft = skb_cuda.FFTProvider(w)
    spec = fft.forward(skb_cuda.make_fixture(w, "sinusoid", 130))
    keep = spec.copy()
    fft.inverse(spec)
    assert np.array_equal(spec, keep)
    assert fft.info()["destroys_native_input"] == 0


def test_fft_split_forms():
    w = skb_cuda.Workload(32, 32, 3, 2)
    real = skb_cuda.make_fixture(w, "random", 131)
    fft = skb_cuda.FFTProvider(w)
    spec = fft.forward(real)
    re, im = fft.forward_split(real)
    assert np.array_equal(re + 1j * im, spec)
    assert np.array_equal(fft.inverse_split(re, im), fft.inverse(spec))


def test_gather_embed_match_reference(golden_vectors):
    g = golden_vectors
    w = skb_cuda.Workload(8, 8, 7, 2)
    fft = skb_cuda.FFTProvider(w)
    for i in range(5):
        ret = fft.gather_retained(g[f"smoke_{i}_spectrum"])
        assert np.array_equal(ret, g[f"smoke_{i}_retained"])
        assert np.array_equal(fft.embed_retained(ret), g[f"smoke_{i}_embedded"])
        re, im = fft.gather_retained_to_split(g[f"smoke_{i}_spectrum"], scale=0.5)
        assert np.array_equal(re + 1j * im, 0.5 * g[f"smoke_{i}_retained"])
        assert np.array_equal(fft.embed_retained_from_split(re * 2, im * 2), g[f"smoke_{i}_embedded"])


def test_fft_fp32_error_against_fp64():
    w = skb_cuda.Workload(256, 256, 9, 2)
    real = skb_cuda.make_fixture(w, "random", 129)
    spec = skb_cuda.FFTProvider(w, skb_cuda.FP32).forward(real)
    assert orc.rel_l2_error(spec, orc.fft_r2c(ow(w), real)) <= 1e-5


# ------------------------------------------------------------------ pruned

def test_pruned_matches_direct_retained(golden_vectors):
    # tests/skbench_tests.cpp ~1290-1575: pruned providers versus directR2C/C2R.
    g = golden_vectors
    for prefix, shape in (("smoke_2", (8, 8, 7, 2)), ("d32", (32, 32, 3, 2))):
        w = skb_cuda.Workload(*shape)
        pr = skb_cuda.PrunedProvider(w)
        ret = pr.forward(g[prefix + "_real"])
        assert orc.max_rel_error(ret, g[prefix + "_retained"]) <= TOL
        assert orc.rel_l2_error(ret, g[prefix + "_retained"]) <= TOL
    w = skb_cuda.Workload(32, 32, 3, 2)
    pr = skb_cuda.PrunedProvider(w)
    out = pr.inverse(g["d32_retained"])
    assert orc.max_rel_error(out, g["d32_embedded_c2r"]) <= TOL


@pytest.mark.parametrize("kind", range(5))
def test_pruned_all_fixtures_smoke(golden_vectors, kind):
    g = golden_vectors
    w = skb_cuda.Workload(8, 8, 7, 2)
    pr = skb_cuda.PrunedProvider(w)
    ret = pr.forward(g[f"smoke_{kind}_real"])
    assert orc.max_rel_error(ret, g[f"smoke_{kind}_retained"]) <= TOL
    out = pr.inverse(g[f"smoke_{kind}_retained"])
    expected = orc.direct_c2r(ow(w), g[f"smoke_{kind}_embedded"])
    assert orc.max_rel_error(out, expected) <= TOL


def test_pruned_quick_profile_matches_full_retained():
    w = skb_cuda.Workload(256, 256, 65, 3)
    real = skb_cuda.make_fixture(w, "random", 129)
    modes = orc.retained_modes(256, 256)
    pr = skb_cuda.PrunedProvider(w)
    info = pr.info()
    assert info["active_kx"] == 86 and info["full_kx"] == 129
    ret = pr.forward(real)
    expected = orc.gather_retained(ow(w), modes, orc.fft_r2c(ow(w), real))
    assert orc.max_rel_error(ret, expected) <= TOL
    assert orc.rel_l2_error(ret, expected) <= TOL
    out = pr.inverse(expected)
    ref = orc.fft_c2r(ow(w), orc.embed_retained(ow(w), modes, expected))
    assert orc.max_rel_error(out, ref) <= TOL


def test_pruned_split_scale_and_field_views():
    w = skb_cuda.Workload(64, 64, 5, 3)
    real = skb_cuda.make_fixture(w, "random", 701)
    pr = skb_cuda.PrunedProvider(w)
    ret = pr.forward(real)
    re, im = pr.forward_split(real, scale=0.25)
    assert np.allclose(re + 1j * im, 0.25 * ret, rtol=0, atol=1e-13 * np.abs(ret).max())
    assert orc.max_rel_error(pr.inverse_split(re * 4, im * 4), pr.inverse(ret)) <= TOL
    # Field views with a mode stride wider than Nz (FFTWStreamingPrunedSplitProvider).
    H, nz, stride = pr.modes, w.nz, w.nz + 3
    fields = [(np.zeros(H * stride), np.zeros(H * stride), stride) for _ in range(w.fields)]
    pr.forward_split_fields(real, fields, scale=1.0)
    comp = ret.reshape(H, w.fields, nz)
    for f, (fr, fi, s) in enumerate(fields):
        got = (fr + 1j * fi).reshape(H, stride)[:, :nz]
        assert orc.max_rel_error(got, comp[:, f, :]) <= TOL
        assert np.all(fr.reshape(H, stride)[:, nz:] == 0)
    out = pr.inverse_split_fields(fields)
    assert orc.max_rel_error(out, pr.inverse(ret)) <= TOL


def test_pruned_field_view_validation():
    w = skb_cuda.Workload(16, 16, 3, 2)
    pr = skb_cuda.PrunedProvider(w)
    real = np.zeros(w.real_elements)
    with pytest.raises(ValueError):
        pr.forward_split_fields(real, [(np.zeros(100), np.zeros(100), 2)] * 2)
    with pytest.raises(ValueError):
        pr.forward_split_fields(real, [(np.zeros(100), np.zeros(100), 3)])


def test_pruned_512_fp32_and_fp64():
    w = skb_cuda.Workload(512, 512, 6, 2)
    real = skb_cuda.make_fixture(w, "random", 702)
    modes = orc.retained_modes(512, 512)
    expected = orc.gather_retained(ow(w), modes, orc.fft_r2c(ow(w), real))
    ret64 = skb_cuda.PrunedProvider(w).forward(real)
    assert orc.rel_l2_error(ret64, expected) <= TOL
    p32 = skb_cuda.PrunedProvider(w, skb_cuda.FP32)
    assert p32.info()["active_kx"] == 171
    assert orc.rel_l2_error(p32.forward(real), expected) <= 1e-5
    back = orc.fft_c2r(ow(w), orc.embed_retained(ow(w), modes, expected))
    assert orc.rel_l2_error(p32.inverse(expected), back) <= 1e-5
