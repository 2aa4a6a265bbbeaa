"""GPU parity of the spectral-pipeline round trip against the reference's own
functions composed in its order (golden vectors) and the oracle at larger sizes:
FP64 at 1e-12, FP32 transforms with TF32x3 GEMMs at 1e-5 relative L2."""

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_weights_match_reference(golden_vectors):
    w = skb_cuda.Workload(16, 16, 9, 2)
    assert np.array_equal(skb_cuda.modal_weights(w), golden_vectors["pipeline_weights"])


def test_fp64_matches_reference_composition(golden_vectors):
    g = golden_vectors
    p = skb_cuda.SpectralPipeline(skb_cuda.Workload(16, 16, 9, 2))
    out = p.execute(g["pipeline_in"])
    assert orc.max_rel_error(out, g["pipeline_out"]) <= 1e-12
    assert orc.rel_l2_error(out, g["pipeline_out"]) <= 1e-12


@pytest.mark.parametrize("shape", [(64, 17, 3), (128, 33, 2)])
def test_against_oracle(shape):
    n, nz, f = shape
    w = skb_cuda.Workload(n, n, nz, f)
    ow = orc.Workload(n, n, nz, f)
    x = orc.make_fixture(ow, 2, 133)
    want = orc.spectral_pipeline(ow, x, workers=8)
    got64 = skb_cuda.SpectralPipeline(w, skb_cuda.FP64).execute(x)
    assert orc.max_rel_error(got64, want) <= 1e-12
    got32 = skb_cuda.SpectralPipeline(w, skb_cuda.FP32).execute(x)
    assert orc.rel_l2_error(got32, want) <= 1e-5


def test_device_form_and_profile():
    w = skb_cuda.Workload(64, 64, 17, 3)
    p = skb_cuda.SpectralPipeline(w)
    x = np.random.default_rng(1).uniform(-1, 1, w.real_elements)
    d_in = skb_cuda.DeviceArray.from_numpy(x)
    d_out = skb_cuda.DeviceArray(x.nbytes)
    p.execute_device(d_in.ptr, d_out.ptr)
    skb_cuda.synchronize()
    assert np.array_equal(d_out.download(np.float64, x.size), p.execute(x))
    stages = p.profile(d_in.ptr, d_out.ptr)
    assert [s["name"] for s in stages] == ["pruned_forward", "vertical_forward", "modal_work", "vertical_inverse",
                                           "pruned_inverse"]
    assert all(s["ms"] > 0 for s in stages)
