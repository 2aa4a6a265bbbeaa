"""GPU parity of the composed 15 -> 4 flux against the reference-composed
golden vectors and the pinned oracle."""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("nz", [7, 13])
def test_flux_fp64_matches_reference(golden_vectors, nz):
    g = golden_vectors
    flux = skb_cuda.Flux(16, nz)
    out = flux.execute(g[f"flux16_{nz}_in"])
    ref = g[f"flux16_{nz}_out"]
    assert orc.max_rel_error(out, ref) <= TOL
    assert orc.rel_l2_error(out, ref) <= TOL


def test_flux_members_and_oracle_64():
    n, nz, members = 64, 17, 3
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    inputs = [orc.flux_inputs(modes, 15, nj, 129 + m) for m in range(members)]
    flux = skb_cuda.Flux(n, nz, members=members)
    out = flux.execute(np.concatenate(inputs)).reshape(members, -1)
    for m in range(members):
        ref = orc.flux(n, nz, inputs[m])
        assert orc.rel_l2_error(out[m], ref) <= TOL
        assert orc.max_rel_error(out[m], ref) <= TOL
    single = skb_cuda.Flux(n, nz).execute(inputs[1])
    assert np.array_equal(single, out[1])


def test_flux_twelve_to_three():
    n, nz = 32, 9
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    x = orc.flux_inputs(modes, 12, nj, 5)
    out = skb_cuda.Flux(n, nz, targets=3).execute(x)
    assert orc.rel_l2_error(out, orc.flux(n, nz, x, targets=3)) <= TOL


def test_flux_fp32_error_against_fp64():
    n, nz = 64, 17
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    x = orc.flux_inputs(modes, 15, nj, 129)
    ref = orc.flux(n, nz, x)
    out = skb_cuda.Flux(n, nz, mode=skb_cuda.FLUX_FP32).execute(x)
    assert orc.rel_l2_error(out, ref) <= 1e-5


def test_flux_graph_replay_equals_direct():
    n, nz = 32, 9
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    x = orc.flux_inputs(modes, 15, nj, 7)
    flux = skb_cuda.Flux(n, nz)
    din = skb_cuda.DeviceArray.from_numpy(x)
    dout = skb_cuda.DeviceArray(flux.output_elements * 16)
    flux.execute_device(din.ptr, dout.ptr)
    skb_cuda.synchronize()
    direct = dout.download(np.complex128, flux.output_elements)
    flux.capture_graph(din.ptr, dout.ptr)
    flux.replay_graph()
    skb_cuda.synchronize()
    assert np.array_equal(dout.download(np.complex128, flux.output_elements), direct)


def test_flux_tf32x3_error_against_fp64():
    n, nz, members = 64, 17, 2
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    xs = [orc.flux_inputs(modes, 15, nj, 129 + m) for m in range(members)]
    out = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3).execute(np.concatenate(xs))
    out = out.reshape(members, -1)
    for m in range(members):
        assert orc.rel_l2_error(out[m], orc.flux(n, nz, xs[m])) <= 1e-6


def test_flux_tf32x3_full_size_against_fp64_cuda():
    # 512x512, Nz=129, 4 targets, 2 members: split precision versus the
    # FP64-plain CUDA path on the same inputs (1e-6).
    n, nz, members = 512, 129, 2
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    x = np.concatenate([orc.flux_inputs(modes, 15, nj, 300 + m) for m in range(members)])
    ref = skb_cuda.Flux(n, nz, members=members).execute(x)
    fast = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_TF32X3)
    out = fast.execute(x)
    fast.check_device()
    assert orc.rel_l2_error(out, ref) <= 1e-6


def test_flux_bf16x3_error_against_oracle():
    # Split BF16x3 tensor-core GEMMs in the fused flux, two members.
    n, nz, members = 64, 17, 2
    modes = orc.retained_modes(n, n)
    nj = 2 * (nz - 1) // 3
    xs = [orc.flux_inputs(modes, 15, nj, 151 + m) for m in range(members)]
    flux = skb_cuda.Flux(n, nz, members=members, mode=skb_cuda.FLUX_SPLIT_BF16X3)
    out = flux.execute(np.concatenate(xs)).reshape(members, -1)
    flux.check_device()
    for m in range(members):
        assert orc.rel_l2_error(out[m], orc.flux(n, nz, xs[m])) <= 1e-6
