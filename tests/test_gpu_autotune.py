"""The project autotuner on the GPU: tuned launch shapes keep the split flux
within its tolerance (1e-6 relative L2 against the FP64-plain path), choices
are cached per shape and reused by later handles, and every band-column form
the tuner may pick at 512 points is correct."""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _inputs(flux, seed):
    rng = np.random.default_rng(seed)
    n = flux.input_elements
    return (rng.uniform(-0.125, 0.125, n) + 1j * rng.uniform(-0.125, 0.125, n)).astype(np.complex64)


def _run(flux, x):
    d_in = skb_cuda.DeviceArray.from_numpy(x)
    d_out = skb_cuda.DeviceArray(flux.output_elements * 8)
    flux.execute_device(d_in.ptr, d_out.ptr)
    skb_cuda.synchronize()
    return d_out.download(np.complex64, flux.output_elements)


def _fp64(n, nz, members, x):
    ref = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_FP64_PLAIN)
    return ref.execute(x.astype(np.complex128))


def test_autotune_keeps_parity_and_caches():
    skb_cuda.tune_cache_clear()
    n, nz, members = 64, 17, 2
    flux = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    x = _inputs(flux, 5)
    d_in = skb_cuda.DeviceArray.from_numpy(x)
    d_out = skb_cuda.DeviceArray(flux.output_elements * 8)
    flux.capture_graph(d_in.ptr, d_out.ptr)
    chosen = flux.autotune(d_in.ptr, d_out.ptr)
    kinds = sorted(" ".join(k.split(" ")[:2]) for k in chosen)
    assert kinds == ["flux.rows.planes_per_cta n=64", "flux.tc_gemm.unit_tiles forward",
                     "flux.tc_gemm.unit_tiles inverse"]
    for key, (value, ms) in chosen.items():
        allowed = (4, 8, 16) if key.startswith("flux.rows") else (4, 8, 16, 32)
        assert value in allowed and ms > 0
    tuned_out = d_out.download(np.complex64, flux.output_elements)
    want = _fp64(n, nz, members, x)
    assert orc.rel_l2_error(tuned_out, want) <= 1e-6
    # The captured graph held the old shapes and was dropped.
    with pytest.raises(skb_cuda.LogicError):
        flux.replay_graph()
    # Cached: a new handle starts with the choices and re-tuning measures nothing.
    for key, (value, _) in chosen.items():
        assert skb_cuda.tune_cache_lookup(key) == value
    again = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    assert {k: v[0] for k, v in again.autotune(d_in.ptr, d_out.ptr).items()} == {k: v[0] for k, v in chosen.items()}
    assert orc.rel_l2_error(_run(again, x), want) <= 1e-6


@pytest.mark.parametrize("mode", [skb_cuda.FLUX_SPLIT_TF32X3, skb_cuda.FLUX_SPLIT_BF16X3], ids=["tf32x3", "bf16x3"])
@pytest.mark.parametrize("tiles", [4, 32])
def test_every_unit_size_is_correct(tiles, mode):
    """A cached choice is applied when a handle is created: force each extreme."""
    skb_cuda.tune_cache_clear()
    n, nz, members = 64, 17, 3
    probe = skb_cuda.Flux(n, nz, members=members, mode=mode)
    x = _inputs(probe, 11)
    d_in = skb_cuda.DeviceArray.from_numpy(x)
    d_out = skb_cuda.DeviceArray(probe.output_elements * 8)
    keys = [k for k in probe.autotune(d_in.ptr, d_out.ptr) if k.startswith("flux.tc_gemm.unit_tiles")]
    assert len(keys) == 2
    for key in keys:
        skb_cuda.tune_cache_store(key, tiles, 0.0)
    flux = skb_cuda.Flux(n, nz, members=members, mode=mode)
    assert orc.rel_l2_error(_run(flux, x), _fp64(n, nz, members, x)) <= 1e-6
    skb_cuda.tune_cache_clear()


@pytest.mark.parametrize("form", [0, 1, 2, 3, 4, 5, 6, 7, 8])
def test_band_forms_at_512(form):
    """Every 512-point band-column kernel form (direct, warp-per-plane,
    persistent direct, direct at four CTAs per SM, direct with 16 or 32 planes
    per CTA, and the 16-plane form walking 16, 32 or 64 columns per CTA) the
    tuner chooses between gives the split flux within 1e-6 of FP64."""
    skb_cuda.tune_cache_clear()
    n, nz, members = 512, 9, 1
    probe = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    x = _inputs(probe, 23)
    d_in = skb_cuda.DeviceArray.from_numpy(x)
    d_out = skb_cuda.DeviceArray(probe.output_elements * 8)
    chosen = probe.autotune(d_in.ptr, d_out.ptr)
    band = [k for k in chosen if k.startswith("flux.columns_band.form")]
    assert len(band) == 2
    for key in band:
        skb_cuda.tune_cache_store(key, form, 0.0)
    flux = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    assert orc.rel_l2_error(_run(flux, x), _fp64(n, nz, members, x)) <= 1e-6
    skb_cuda.tune_cache_clear()


@pytest.mark.parametrize("n,planes,pairs,tma", [(64, 4, 0, 0), (64, 16, 0, 0), (512, 4, 0, 0), (512, 16, 0, 0),
                                                (512, 8, 1, 0), (512, 16, 1, 0), (512, 8, 2, 0), (512, 8, 1, 1),
                                                (512, 16, 1, 1), (512, 8, 2, 1), (512, 24, 1, 0),
                                                (512, 8, 2, 2), (512, 16, 1, 2)])
def test_every_row_kernel_width_is_correct(n, planes, pairs, tma):
    """The fused row kernel with 4, 8 or 16 z-planes per CTA, and at 512 points
    the two-planes-per-warp form with 8, 16 or 24, its stages filled by
    cp.async or by TMA tensor copies one or two slots ahead (the tuner's
    candidates)."""
    skb_cuda.tune_cache_clear()
    nz, members = 17, 2
    probe = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    x = _inputs(probe, 31)
    d_in = skb_cuda.DeviceArray.from_numpy(x)
    d_out = skb_cuda.DeviceArray(probe.output_elements * 8)
    chosen = probe.autotune(d_in.ptr, d_out.ptr)
    keys = [k for k in chosen if k.startswith("flux.rows.planes_per_cta")]
    assert len(keys) == 1
    skb_cuda.tune_cache_store(keys[0], planes, 0.0)
    pair_keys = [k for k in chosen if k.startswith("flux.rows.pairs")]
    assert len(pair_keys) == (1 if n == 512 else 0)
    for key in pair_keys:
        skb_cuda.tune_cache_store(key, pairs, 0.0)
        skb_cuda.tune_cache_store(key.replace("flux.rows.pairs", "flux.rows.tma", 1), tma, 0.0)
    flux = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    assert orc.rel_l2_error(_run(flux, x), _fp64(n, nz, members, x)) <= 1e-6
    flux.check_device()
    skb_cuda.tune_cache_clear()


def test_row_kernel_expired_wait_is_reported_and_the_context_survives():
    """The fused row kernel's TMA forms bound the wait for each stage copy:
    with the test flag, thread 0 also waits on a barrier nothing signals, the
    wait runs out, the flux reports SKB_ERR_RUNTIME instead of hanging, and a
    new handle on the same context computes correctly."""
    import ctypes

    skb_cuda.tune_cache_clear()
    n, nz, members = 512, 9, 1
    probe = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    x = _inputs(probe, 41)
    d_in = skb_cuda.DeviceArray.from_numpy(x)
    d_out = skb_cuda.DeviceArray(probe.output_elements * 8)
    chosen = probe.autotune(d_in.ptr, d_out.ptr)
    probe.close()
    pair_keys = [k for k in chosen if k.startswith("flux.rows.pairs ")]
    assert len(pair_keys) == 1
    skb_cuda.tune_cache_store(pair_keys[0], 2, 0.0)
    skb_cuda.tune_cache_store(pair_keys[0].replace("flux.rows.pairs", "flux.rows.tma", 1), 1, 0.0)
    skb_cuda.tune_cache_store(pair_keys[0].replace("flux.rows.pairs", "flux.rows.planes_per_cta", 1), 8, 0.0)
    flux = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    skb_cuda.check(skb_cuda.library().skb_flux_rows_expire_wait_for_test(flux.h, ctypes.c_int(1)))
    _run(flux, x)
    with pytest.raises(RuntimeError, match="bounded wait"):
        flux.check_device()
    flux.close()
    fresh = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    assert orc.rel_l2_error(_run(fresh, x), _fp64(n, nz, members, x)) <= 1e-6
    fresh.check_device()
    skb_cuda.tune_cache_clear()
