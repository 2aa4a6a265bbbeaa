"""GPU parity of the authoritative two-family flux (wave-f / wave-g operators
over floating groups, loaded from a prepared fixture) against the fixture's
expected targets, which the oracle's two-family flux computed: FP64-plain at
1e-12 (the reference's authoritative tolerance), split TF32x3 at 1e-6."""

import numpy as np
import pytest

import skb_cuda
import skb_cuda.fixture as fx
from oracle import oracle as orc
from synthetic_fixture import make

pytestmark = pytest.mark.gpu


def _families(f):
    return {"group_modes": f.group_modes, "forward": f.forward, "inverse": f.inverse,
            "input_family": f.input_family, "target_family": f.target_family}


@pytest.mark.parametrize("n,nz,mode,tol", [
    (16, 9, skb_cuda.FLUX_FP64_PLAIN, 1e-12),
    (16, 9, skb_cuda.FLUX_SPLIT_TF32X3, 1e-6),   # staged path, tensor-core GEMMs on field subsets
    (64, 17, skb_cuda.FLUX_FP64_PLAIN, 1e-12),
    (64, 17, skb_cuda.FLUX_SPLIT_TF32X3, 1e-6),  # fused dense path
])
def test_fixture_flux_matches_expected(tmp_path, n, nz, mode, tol):
    path = tmp_path / "fixture.bin"
    make(path, n, nz)
    f = fx.load(path)
    flux = skb_cuda.Flux(n, nz, members=1, mode=mode, families=_families(f))
    got = flux.execute(f.modal_inputs.reshape(-1)).reshape(f.expected_targets.shape)
    err = orc.rel_l2_error(got, f.expected_targets)
    assert err <= tol, err
    if mode == skb_cuda.FLUX_FP64_PLAIN:
        assert orc.max_rel_error(got, f.expected_targets) <= tol


def test_members_are_independent(tmp_path):
    """Two members with different inputs through one two-family handle."""
    n, nz = 64, 17
    path = tmp_path / "fixture.bin"
    make(path, n, nz, seed=11)
    f = fx.load(path)
    fam = _families(f)
    x2 = f.modal_inputs * (0.5 - 0.25j)
    x2[0].imag = 0.0
    want2 = orc.flux(n, nz, x2.reshape(-1), families=fam).reshape(f.expected_targets.shape)
    for mode, tol in ((skb_cuda.FLUX_FP64_PLAIN, 1e-12), (skb_cuda.FLUX_SPLIT_TF32X3, 1e-6)):
        flux = skb_cuda.Flux(n, nz, members=2, mode=mode, families=fam)
        got = flux.execute(np.concatenate([f.modal_inputs.reshape(-1), x2.reshape(-1)])).reshape(2, -1)
        assert orc.rel_l2_error(got[0], f.expected_targets) <= tol
        assert orc.rel_l2_error(got[1], want2) <= tol


def test_bad_families_are_refused():
    with pytest.raises(ValueError):
        skb_cuda.Flux(16, 9, families={"group_modes": np.array([1], np.uint64), "forward": [np.zeros(45)] * 2,
                                       "inverse": [np.zeros(45)] * 2, "input_family": fx.INPUT_FAMILIES,
                                       "target_family": fx.TARGET_FAMILIES})


@pytest.mark.parametrize("mode,tol", [(skb_cuda.FLUX_FP64_PLAIN, 1e-12), (skb_cuda.FLUX_SPLIT_TF32X3, 1e-6)])
def test_golden_fixture_matches_the_reference_composition(golden_vectors, mode, tol):
    """The golden prepared fixture (read by the reference's own loader when it
    was made) against the two-family flux composed from the reference's
    functions: FP64-plain at the reference's 1e-12, split TF32x3 at 1e-6."""
    import os

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "two_family_16x7.skfxp")
    f = fx.load(path)
    ref = golden_vectors["two_family_targets"]
    for members in (1, 2):
        flux = skb_cuda.Flux(f.nx, f.nz, members=members, mode=mode, families=_families(f))
        x = np.concatenate([f.modal_inputs.reshape(-1)] * members)
        got = flux.execute(x).reshape(members, *ref.shape)
        for m in range(members):
            assert orc.max_rel_error(got[m], ref) <= tol
            assert orc.rel_l2_error(got[m], ref) <= tol
        flux.close()
