"""The C-ABI boundary on CPU: symbol table, host-side model, loud failures.

No compute call here touches a GPU; these run in the CPU suite.
"""

import ctypes
import hashlib
import os
import re

import numpy as np
import pytest

import skb_cuda
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for header in os.listdir(os.path.join(ROOT, "include")):
        if header.endswith(".h"):
            text = open(os.path.join(ROOT, "include", header)).read()
            names |= set(re.findall(r"^SKB_API\s+[\w\s\*]*?\b(skb_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 80
    lib = skb_cuda.library()
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert "sm_100a" in skb_cuda.version()


@pytest.mark.parametrize("n,nz,f", [(8, 7, 2), (16, 7, 2), (128, 33, 3), (256, 65, 3), (512, 129, 4)])
def test_model_known_answers(known_answers, n, nz, f):
    case = next(c for c in known_answers["known_answers"] if (c["n"], c["nz"], c["fields"]) == (n, nz, f))
    w = skb_cuda.Workload(n, n, nz, f)
    modes = skb_cuda.retained_modes(w)
    groups = skb_cuda.squared_wavenumber_groups(w)
    assert len(modes) == case["modes"]
    assert len(groups) == case["groups"]
    mh, gh, wh = skb_cuda.order_hashes(w, wvm=n <= 256)
    assert mh == case["mode_hash"] and gh == case["group_hash"]
    if n <= 256:
        assert wh == case["wvm_hash"]


def test_model_modes_match_oracle_bitwise():
    for n in (8, 32, 256):
        mine = skb_cuda.retained_modes(skb_cuda.Workload(n, n, 7, 1))
        ref = orc.retained_modes(n, n)
        assert [m.k for m in mine] == list(ref.k)
        assert [m.l for m in mine] == list(ref.l)
        assert [m.stored_kx for m in mine] == list(ref.kx)
        assert [m.stored_ky for m in mine] == list(ref.ky)
        assert [bool(m.conjugates_stored_value) for m in mine] == list(ref.conj)
        assert np.array_equal(np.array([m.radial_mode for m in mine]), ref.radial)


def test_fixture_generator_matches_reference(known_answers, golden_vectors):
    for case in known_answers["fixture_sha256"]:
        w = skb_cuda.Workload(case["n"], case["n"], case["nz"], case["fields"])
        v = skb_cuda.make_fixture(w, case["kind"], case["seed"])
        assert hashlib.sha256(v.tobytes()).hexdigest() == case["sha256"]
    w = skb_cuda.Workload(8, 8, 7, 2)
    for i in range(5):
        assert np.array_equal(skb_cuda.make_fixture(w, i, 129 + i), golden_vectors[f"smoke_{i}_real"])


def test_vertical_families_match_reference(golden_vectors, known_answers):
    fwd, inv, ident = skb_cuda.vertical_family(skb_cuda.Workload(16, 16, 9, 3), skb_cuda.FAMILY_K2_ROTATION)
    assert ident == known_answers["k2_family_id"]
    assert np.array_equal(fwd, golden_vectors["k2_forward"])
    assert np.array_equal(inv, golden_vectors["k2_inverse"])
    fwd, inv, ident = skb_cuda.vertical_family(skb_cuda.Workload(8, 8, 7, 2), skb_cuda.FAMILY_COMMON_DCT2)
    assert ident == "orthonormal-dct2-truncated-v1"
    assert np.array_equal(fwd, golden_vectors["smoke_vertical_forward"])
    assert np.array_equal(inv, golden_vectors["smoke_vertical_inverse"])


def test_sturm_liouville_family_is_orthonormal_and_group_dependent():
    w = skb_cuda.Workload(32, 32, 17, 3)
    fwd, inv, ident = skb_cuda.vertical_family(w, skb_cuda.FAMILY_STURM_LIOUVILLE, seed=129)
    nj, nz = w.nj, w.nz
    F = fwd.reshape(-1, nj, nz)
    I = inv.reshape(-1, nz, nj)
    assert ident.startswith("seeded-sturm-liouville")
    for g in (0, len(F) // 2, len(F) - 1):
        assert np.allclose(F[g] @ F[g].T, np.eye(nj), atol=1e-10)
        assert np.array_equal(I[g], F[g].T)
    assert not np.allclose(F[1], F[-1])


def test_invalid_arguments_raise_value_error():
    with pytest.raises(ValueError):
        skb_cuda.retained_modes(skb_cuda.Workload(1, 8, 7, 2))
    with pytest.raises(ValueError):
        skb_cuda.make_fixture(skb_cuda.Workload(8, 8, 0, 2), 2, 1)


def test_gpu_calls_fail_loudly_without_a_device():
    if skb_cuda_has_device():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        skb_cuda.FFTProvider(skb_cuda.Workload(8, 8, 7, 2))


def skb_cuda_has_device():
    try:
        return skb_cuda.device_count() > 0
    except RuntimeError:
        return False
