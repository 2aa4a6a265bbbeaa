"""GPU parity of the K^2-grouped vertical GEMM and the pointwise product."""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-12


def provider(w, layout=skb_cuda.INTERLEAVED, policy=skb_cuda.BIDIRECTIONAL, precision=skb_cuda.GEMM_FP64,
             family=skb_cuda.FAMILY_K2_ROTATION):
    groups = skb_cuda.squared_wavenumber_groups(w)
    fwd, inv, _ = skb_cuda.vertical_family(w, family)
    if family == skb_cuda.FAMILY_COMMON_DCT2:
        groups = [skb_cuda.ModeGroup(0, 0, sum(g.mode_count for g in groups))]
    return skb_cuda.VerticalGemmProvider(w, groups, fwd, inv, layout, policy, precision)


def test_k2_grouped_matches_reference_projections(golden_vectors):
    g = golden_vectors
    w = skb_cuda.Workload(16, 16, 9, 3)
    vp = provider(w)
    vp.load_physical_input(g["k2_phys"])
    vp.execute_forward()
    assert orc.max_rel_error(vp.copy_forward_output(), g["k2_modal"]) <= TOL
    vp.load_modal_input(g["k2_modal_in"])
    vp.execute_inverse()
    assert orc.max_rel_error(vp.copy_inverse_output(), g["k2_phys_out"]) <= TOL


def test_split_layout_matches_interleaved(golden_vectors):
    g = golden_vectors
    w = skb_cuda.Workload(16, 16, 9, 3)
    vp = provider(w, layout=skb_cuda.SPLIT)
    vp.load_physical_input_split(g["k2_phys"].real, g["k2_phys"].imag)
    vp.execute_forward()
    re, im = vp.copy_forward_output_split()
    assert orc.max_rel_error(re + 1j * im, g["k2_modal"]) <= TOL
    with pytest.raises(skb_cuda.LogicError):
        vp.copy_forward_output()


def test_buffer_policies_reject_wrong_direction():
    w = skb_cuda.Workload(16, 16, 9, 3)
    fwd_only = provider(w, policy=skb_cuda.FORWARD_ONLY)
    with pytest.raises(skb_cuda.LogicError):
        fwd_only.execute_inverse()
    inv_only = provider(w, policy=skb_cuda.INVERSE_ONLY)
    with pytest.raises(skb_cuda.LogicError):
        inv_only.execute_forward()


@pytest.mark.parametrize("shape", [(256, 256, 65, 3), (128, 128, 33, 4)])
def test_k2_grouped_matches_oracle(shape):
    w = skb_cuda.Workload(*shape)
    o = orc.Workload(*shape)
    fam = orc.k2_family(o)
    H = len(orc.retained_modes(w.nx, w.ny))
    rng = np.random.default_rng(11)
    phys = rng.uniform(-1, 1, H * w.fields * w.nz) + 1j * rng.uniform(-1, 1, H * w.fields * w.nz)
    modal = rng.uniform(-1, 1, H * w.fields * w.nj) + 1j * rng.uniform(-1, 1, H * w.fields * w.nj)
    vp = provider(w)
    vp.load_physical_input(phys)
    vp.execute_forward()
    got = vp.copy_forward_output()
    ref = orc.grouped_vertical(o, fam, "forward", phys)
    assert orc.max_rel_error(got, ref) <= TOL and orc.rel_l2_error(got, ref) <= TOL
    vp.load_modal_input(modal)
    vp.execute_inverse()
    got = vp.copy_inverse_output()
    ref = orc.grouped_vertical(o, fam, "inverse", modal)
    assert orc.max_rel_error(got, ref) <= TOL and orc.rel_l2_error(got, ref) <= TOL
    # FP32 SIMT form against the FP64 oracle.
    v32 = provider(w, precision=skb_cuda.GEMM_FP32)
    v32.load_modal_input(modal)
    v32.execute_inverse()
    assert orc.rel_l2_error(v32.copy_inverse_output(), ref) <= 1e-6


def test_common_family_matches_vertical_forward(golden_vectors):
    # verticalForward with the common DCT-II operator (validate, benchmark.cpp:4985-4995).
    g = golden_vectors
    w = skb_cuda.Workload(8, 8, 7, 2)
    vp = provider(w, family=skb_cuda.FAMILY_COMMON_DCT2)
    for i in range(5):
        ret = g[f"smoke_{i}_retained"]
        vp.load_physical_input(ret)
        vp.execute_forward()
        modal = vp.copy_forward_output()
        F = g["smoke_vertical_forward"].reshape(w.nj, w.nz)
        ref = (ret.reshape(-1, w.nz) @ F.T).reshape(-1)
        assert orc.max_rel_error(modal, ref) <= TOL
        vp.load_modal_input(modal)
        vp.execute_inverse()
        again = vp.copy_inverse_output()
        vp.load_physical_input(again)
        vp.execute_forward()
        assert orc.max_rel_error(vp.copy_forward_output(), modal) <= TOL


def test_pointwise_matches_reference(golden_vectors):
    # tests/skbench_tests.cpp:1136-1185 at 1e-15.
    g = golden_vectors
    ex = skb_cuda.PointwiseAdvectionExecutor(37, 0.03125)
    out = ex.execute(g["pointwise_shared"], g["pointwise_derivative"])
    assert orc.max_rel_error(out, g["pointwise_0"]) <= 1e-15


def test_pointwise_large_volume():
    n = 64 * 64 * 17 + 1
    rng = np.random.default_rng(4)
    s = rng.standard_normal(3 * n)
    d = rng.standard_normal(3 * n)
    scale = 1.0 / (64.0 * 64.0) ** 2
    out = skb_cuda.PointwiseAdvectionExecutor(n, scale).execute(s, d)
    ref = orc.pointwise(n, scale, s, d)
    assert orc.max_rel_error(out, ref) <= 1e-15
    out32 = skb_cuda.PointwiseAdvectionExecutor(n, scale, skb_cuda.FP32).execute(s, d)
    assert orc.rel_l2_error(out32, ref) <= 1e-6


# ------------------------------------------------------- tensor-core form

@pytest.mark.parametrize("precision", [skb_cuda.GEMM_TF32X3, skb_cuda.GEMM_BF16X3], ids=["tf32x3", "bf16x3"])
@pytest.mark.parametrize("shape", [(16, 16, 9, 3), (16, 16, 7, 2), (256, 256, 65, 3), (128, 128, 33, 4),
                                   (512, 512, 129, 15)])
def test_split_tensor_core_matches_oracle(shape, precision):
    # Split TF32x3 (kind::tf32) and split BF16x3 (kind::f16, three BF16 pieces,
    # six products) on tcgen05 with FP32 accumulation: FP32-level error
    # against FP64.
    w = skb_cuda.Workload(*shape)
    o = orc.Workload(*shape)
    fam = orc.k2_family(o)
    H = len(orc.retained_modes(w.nx, w.ny))
    rng = np.random.default_rng(12)
    phys = rng.uniform(-1, 1, H * w.fields * w.nz) + 1j * rng.uniform(-1, 1, H * w.fields * w.nz)
    modal = rng.uniform(-1, 1, H * w.fields * w.nj) + 1j * rng.uniform(-1, 1, H * w.fields * w.nj)
    vp = provider(w, precision=precision)
    vp.load_physical_input(phys)
    vp.execute_forward()
    got = vp.copy_forward_output()
    ref = orc.grouped_vertical(o, fam, "forward", phys)
    assert orc.rel_l2_error(got, ref) <= 1e-6
    assert orc.max_rel_error(got, ref) <= 2e-6
    vp.load_modal_input(modal)
    vp.execute_inverse()
    got = vp.copy_inverse_output()
    ref = orc.grouped_vertical(o, fam, "inverse", modal)
    assert orc.rel_l2_error(got, ref) <= 1e-6
    assert orc.max_rel_error(got, ref) <= 2e-6


def test_tf32x3_rejects_split_layout():
    w = skb_cuda.Workload(16, 16, 9, 3)
    with pytest.raises(ValueError):
        provider(w, layout=skb_cuda.SPLIT, precision=skb_cuda.GEMM_TF32X3)


def test_tf32x3_expired_wait_is_reported_and_the_context_survives():
    """The tensor-core GEMM's error path: a bounded device wait on a barrier
    that nothing signals runs out; the call reports SKB_ERR_RUNTIME instead of
    hanging, and a new provider on the same context computes correctly."""
    import ctypes

    shape = (64, 64, 17, 2)
    w = skb_cuda.Workload(*shape)
    H = len(orc.retained_modes(w.nx, w.ny))
    rng = np.random.default_rng(3)
    phys = rng.uniform(-1, 1, H * w.fields * w.nz) + 1j * rng.uniform(-1, 1, H * w.fields * w.nz)
    vp = provider(w, precision=skb_cuda.GEMM_TF32X3)
    skb_cuda.check(skb_cuda.library().skb_vertical_expire_wait_for_test(vp.h, ctypes.c_int(1)))
    vp.load_physical_input(phys)
    with pytest.raises(RuntimeError, match="bounded device wait expired"):
        vp.execute_forward()
    vp.close()
    fresh = provider(w, precision=skb_cuda.GEMM_TF32X3)
    fresh.load_physical_input(phys)
    fresh.execute_forward()
    ref = orc.grouped_vertical(orc.Workload(*shape), orc.k2_family(orc.Workload(*shape)), "forward", phys)
    assert orc.rel_l2_error(fresh.copy_forward_output(), ref) <= 1e-6
