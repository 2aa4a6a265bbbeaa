"""The prepared spectral-flux fixture format (the authoritative WVM boundary)
on CPU: loader round trip, the reference's validation rules, and the oracle's
two-family flux against its one-family form."""

import os
import struct
import subprocess

import numpy as np
import pytest

import skb_cuda.fixture as fx
from oracle import oracle as orc
from synthetic_fixture import families_canonical, make


def test_round_trip(tmp_path):
    path = tmp_path / "f.bin"
    fam, inputs, expected = make(path, 16, 9)
    f = fx.load(path)
    assert (f.nx, f.ny, f.nz, f.nj) == (16, 16, 9, 5)
    assert np.array_equal(f.group_modes, fam["group_modes"])
    for d in ("forward", "inverse"):
        for k in range(2):
            assert np.array_equal(getattr(f, d)[k], fam[d][k])
    assert np.array_equal(f.modal_inputs, inputs)
    assert np.array_equal(f.expected_targets, expected)
    assert f.input_family == fx.INPUT_FAMILIES and f.target_family == fx.TARGET_FAMILIES
    assert f.pointwise_scale == 1.0 / 16.0 ** 4


def _corrupt(tmp_path, edit):
    path = tmp_path / "f.bin"
    make(path, 8, 7)
    data = bytearray(path.read_bytes())
    edit(data)
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(data))
    return bad


@pytest.mark.parametrize("edit,message", [
    (lambda d: d.__setitem__(slice(0, 8), b"SKFXP002"), "wrong magic"),
    (lambda d: d.__setitem__(slice(16, 20), struct.pack("<I", 0)), "not authoritative"),
    (lambda d: d.extend(b"\0"), "trailing bytes"),
    (lambda d: d.__delitem__(slice(len(d) - 16, len(d))), "truncated"),
])
def test_validation_rejects(tmp_path, edit, message):
    with pytest.raises(fx.FixtureError, match=message):
        fx.load(_corrupt(tmp_path, edit))


def test_validation_rejects_a_wrong_family_map(tmp_path):
    modes, fam, keys = families_canonical(8, 7, 3)
    H = len(modes)
    path = tmp_path / "f.bin"
    group_of = np.repeat(np.arange(len(fam["group_modes"])), fam["group_modes"].astype(np.int64))
    inputs = np.zeros((H, 15, 4), complex)
    wrong = list(fx.INPUT_FAMILIES)
    wrong[0] = 1
    fx.write(path, 8, 7, np.stack([modes.k, modes.l], 1), group_of, keys, fam["forward"], fam["inverse"], inputs,
             np.zeros((H, 4, 4), complex), input_family=wrong)
    with pytest.raises(fx.FixtureError, match="input field-to-operator map"):
        fx.load(path)


def test_validation_rejects_a_missing_mode(tmp_path):
    modes, fam, keys = families_canonical(8, 7, 3)
    H = len(modes)
    k = np.stack([modes.k, modes.l], 1).copy()
    k[-1] = (99, 99)  # not a retained mode (also breaks its group key)
    group_of = np.repeat(np.arange(len(fam["group_modes"])), fam["group_modes"].astype(np.int64))
    path = tmp_path / "f.bin"
    fx.write(path, 8, 7, k, group_of, keys, fam["forward"], fam["inverse"], np.zeros((H, 15, 4), complex),
             np.zeros((H, 4, 4), complex))
    with pytest.raises(fx.FixtureError, match="missing a retained horizontal mode key"):
        fx.load(path)


CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "spectral-kernel-benchmarks_b200",
                   "skbench-cuda")


def _cli_rejects(path, message):
    out = subprocess.run([CLI, "run", "--kernel", "production-lifetime-flux", "--spectral-flux-fixture", str(path)],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 2, out.stdout + out.stderr
    assert message in out.stderr


@pytest.mark.skipif(not os.path.exists(CLI), reason="skbench-cuda is not built")
@pytest.mark.parametrize("edit,message", [
    (lambda d: d.__setitem__(slice(0, 8), b"SKFXP002"), "wrong magic"),
    (lambda d: d.__setitem__(slice(16, 20), struct.pack("<I", 0)), "not authoritative"),
    (lambda d: d.extend(b"\0"), "trailing bytes"),
    (lambda d: d.__delitem__(slice(len(d) - 16, len(d))), "truncated"),
])
def test_cli_loader_rejects_like_the_python_one(tmp_path, edit, message):
    """The command line's C++ reader (harness/fixture.cpp) applies the same
    checks, before any device work, with the same reasons."""
    bad = _corrupt(tmp_path, edit)
    with pytest.raises(fx.FixtureError, match=message):
        fx.load(bad)
    _cli_rejects(bad, message)


@pytest.mark.skipif(not os.path.exists(CLI), reason="skbench-cuda is not built")
def test_cli_loader_rejects_a_wrong_family_map_and_a_missing_mode(tmp_path):
    modes, fam, keys = families_canonical(8, 7, 3)
    H = len(modes)
    group_of = np.repeat(np.arange(len(fam["group_modes"])), fam["group_modes"].astype(np.int64))
    wrong = list(fx.INPUT_FAMILIES)
    wrong[0] = 1
    path = tmp_path / "map.bin"
    fx.write(path, 8, 7, np.stack([modes.k, modes.l], 1), group_of, keys, fam["forward"], fam["inverse"],
             np.zeros((H, 15, 4), complex), np.zeros((H, 4, 4), complex), input_family=wrong)
    _cli_rejects(path, "input field-to-operator map")
    k = np.stack([modes.k, modes.l], 1).copy()
    k[-1] = (99, 99)
    path = tmp_path / "mode.bin"
    fx.write(path, 8, 7, k, group_of, keys, fam["forward"], fam["inverse"], np.zeros((H, 15, 4), complex),
             np.zeros((H, 4, 4), complex))
    _cli_rejects(path, "missing a retained horizontal mode key")


def test_two_family_oracle_reduces_to_the_one_family_flux():
    """With both families equal to the K^2 family over the K^2 groups, the
    two-family flux is the production flux."""
    n, nz = 16, 9
    w = orc.Workload(n, n, nz, 4)
    fwd, inv = orc.k2_family(w)
    _, _, counts = orc.k2_groups(n, n)
    fam = {"group_modes": counts, "forward": [fwd, fwd], "inverse": [inv, inv],
           "input_family": fx.INPUT_FAMILIES, "target_family": fx.TARGET_FAMILIES}
    rng = np.random.default_rng(2)
    H = len(orc.retained_modes(n, n))
    x = rng.uniform(-0.125, 0.125, H * 15 * 5) + 1j * rng.uniform(-0.125, 0.125, H * 15 * 5)
    a = orc.flux(n, nz, x, families=fam)
    b = orc.flux(n, nz, x)
    assert orc.max_rel_error(a, b) <= 1e-14


@pytest.mark.parametrize("change,message", [
    (lambda fam, o: o.update(targets=3), "15 -> 4"),
    # (matrices padded or emptied to the changed group count, so the C ABI's own
    # checks are the ones that refuse)
    (lambda fam, o: fam.update(group_modes=np.concatenate([[0], fam["group_modes"]]).astype(np.uint64),
                               forward=[np.concatenate([f[:1], f]) for f in fam["forward"]],
                               inverse=[np.concatenate([i[:1], i]) for i in fam["inverse"]]),
     "nonempty"),
    (lambda fam, o: fam.update(group_modes=np.zeros(0, np.uint64), forward=[f[:0] for f in fam["forward"]],
                               inverse=[i[:0] for i in fam["inverse"]]), "operator groups"),
    # Matrices shaped for another Nz or group count, and short family maps, are
    # refused by the binding before the C ABI copies groups * Nj * Nz values.
    (lambda fam, o: fam.update(forward=[f[:, :, :-1] for f in fam["forward"]]), "expected"),
    (lambda fam, o: fam.update(inverse=[i[:-1] for i in fam["inverse"]]), "expected"),
    (lambda fam, o: fam.update(forward=fam["forward"][:1]), "wave-f and wave-g"),
    (lambda fam, o: fam.update(input_family=list(fam["input_family"])[:14]), "15 slots"),
    (lambda fam, o: fam.update(target_family=list(fam["target_family"]) + [0]), "4 slots"),
])
def test_family_flux_arguments_are_refused_before_device_work(change, message):
    """skb_flux_create_families checks its arguments (the reference's
    std::invalid_argument cases) before it allocates anything on a device."""
    import skb_cuda

    _, fam, _ = families_canonical(8, 7, 3)
    opts = {"targets": 4}
    change(fam, opts)
    with pytest.raises(ValueError, match=message):
        skb_cuda.Flux(8, 7, targets=opts["targets"], members=1, mode=skb_cuda.FLUX_FP64_PLAIN, families=fam)


GOLDEN_FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "two_family_16x7.skfxp")


def test_loader_matches_the_reference_loader(golden_vectors):
    """The golden two-family fixture as this library's loader returns it equals,
    bit for bit, what the reference's loadPreparedSpectralFluxFixture made of
    the same file (mode order, operator groups, each group's matrices through
    its source group, inputs and targets)."""
    g = golden_vectors
    f = fx.load(GOLDEN_FIXTURE)
    import skb_cuda

    mine = skb_cuda.retained_modes(skb_cuda.Workload(f.nx, f.ny, f.nz, 4))
    assert [m.k for m in mine] == list(g["two_family_k"])
    assert [m.l for m in mine] == list(g["two_family_l"])
    assert np.array_equal(f.group_modes, g["two_family_group_count"])
    assert np.array_equal(np.r_[0, np.cumsum(f.group_modes)[:-1]], g["two_family_group_first"])
    assert np.array_equal(f.group_keys, g["two_family_group_key"])
    source = g["two_family_matrix_source"].astype(np.int64)
    for fam in range(2):
        assert np.array_equal(f.forward[fam], g["two_family_forward"][fam][source])
        assert np.array_equal(f.inverse[fam], g["two_family_inverse"][fam][source])
    assert np.array_equal(f.modal_inputs, g["two_family_inputs"])
    assert np.array_equal(f.expected_targets, g["two_family_targets"])


def test_two_family_oracle_matches_the_reference_composition(golden_vectors):
    """The oracle's two-family flux against the one composed from the
    reference's own functions (loader, verticalInverse / verticalForward with
    the family maps, direct DFTs, PointwiseAdvectionExecutor) at the
    reference's FP64 tolerance."""
    f = fx.load(GOLDEN_FIXTURE)
    fam = {"group_modes": f.group_modes, "forward": f.forward, "inverse": f.inverse,
           "input_family": f.input_family, "target_family": f.target_family}
    got = orc.flux(f.nx, f.nz, f.modal_inputs.reshape(-1), families=fam)
    ref = golden_vectors["two_family_targets"].reshape(-1)
    assert orc.max_rel_error(got, ref) <= 1e-12
    assert orc.rel_l2_error(got, ref) <= 1e-12
