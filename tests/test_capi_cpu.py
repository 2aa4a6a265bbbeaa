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


@pytest.mark.parametrize("shape,seed", [((32, 32, 17, 3), 129), ((128, 128, 33, 3), 7)])
def test_sturm_liouville_family_matches_lapack_restatement(shape, seed):
    # The library's QL iteration against LAPACK's tridiagonal eigensolver on the
    # same seeded operator: eigenvectors agree to rounding (the spectrum is
    # simple, so the vectors are unique up to the fixed sign convention).
    w = skb_cuda.Workload(*shape)
    fwd, inv, _ = skb_cuda.vertical_family(w, skb_cuda.FAMILY_STURM_LIOUVILLE, seed=seed)
    ofwd, oinv = orc.sturm_liouville_family(orc.Workload(*shape), seed)
    assert np.max(np.abs(fwd.reshape(ofwd.shape) - ofwd)) <= 1e-10
    assert np.max(np.abs(inv.reshape(oinv.shape) - oinv)) <= 1e-10


def test_invalid_arguments_raise_value_error():
    with pytest.raises(ValueError):
        skb_cuda.retained_modes(skb_cuda.Workload(1, 8, 7, 2))
    with pytest.raises(ValueError):
        skb_cuda.make_fixture(skb_cuda.Workload(8, 8, 0, 2), 2, 1)


def test_type1_handle_arguments_are_refused_before_device_work():
    """skb_cs_vertical_create: rows > 0 and Nz in [3, 16385] (a DCT-I needs
    two intervals), checked before any stream or allocation."""
    for rows, nz in ((4, 2), (0, 9), (4, 16386)):
        with pytest.raises(ValueError):
            skb_cuda.ConstantStratificationVertical(rows, nz)


def test_allocation_free_inverse_refuses_an_overflowing_workload():
    # Nz * fields wraps a 64-bit product (2^62 * 8 = 2^65); the scratch size
    # saturates instead, so the call is refused before any device work.
    lib = skb_cuda.library()
    for w in (skb_cuda.Workload(64, 64, 1 << 62, 8), skb_cuda.Workload(1024, 1024, (1 << 64) - 1, 3)):
        with pytest.raises(ValueError, match="bytes of scratch"):
            skb_cuda.check(lib.skb_fft_inverse_device_noalloc(ctypes.byref(w), ctypes.c_int(skb_cuda.FP64),
                                                              ctypes.c_void_p(16), ctypes.c_void_p(16),
                                                              ctypes.c_void_p(None)))


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


def test_tuning_cache_round_trip(tmp_path):
    """The autotuner's cache on the host: store / lookup / save / clear / load,
    one "<value> <ms> <key>" line per entry."""
    skb_cuda.tune_cache_clear()
    key = "flux.tc_gemm.unit_tiles inverse n=64 nz=17 targets=4 members=2 R=17 S=10 groups=40 | test-device/1"
    skb_cuda.tune_cache_store(key, 8, 0.125)
    assert skb_cuda.tune_cache_lookup(key) == 8
    assert skb_cuda.tune_cache_lookup(key + " other") is None
    path = tmp_path / "tune.txt"
    assert skb_cuda.tune_cache_save(str(path)) == 1
    assert path.read_text() == "8 0.125 " + key + "\n"
    skb_cuda.tune_cache_clear()
    assert skb_cuda.tune_cache() == {}
    path.write_text(path.read_text() + "not a line\n16 2.5 second key | test-device/1\n")
    assert skb_cuda.tune_cache_load(str(path)) == 2
    assert skb_cuda.tune_cache() == {key: (8, 0.125), "second key | test-device/1": (16, 2.5)}
    with pytest.raises(ValueError):
        skb_cuda.tune_cache_store("two\nlines", 1)
    skb_cuda.tune_cache_clear()


def test_tuning_cache_file_from_the_environment(tmp_path):
    """SKB_TUNE_CACHE: a new process starts with the file's choices and appends
    the ones it makes."""
    import subprocess
    import sys

    path = tmp_path / "env_tune.txt"
    path.write_text("32 1.5 stage A | test-device/1\n")
    code = ("import sys; sys.path.insert(0, %r); import skb_cuda as S; "
            "print(S.tune_cache_lookup('stage A | test-device/1')); S.tune_cache_store('stage B | test-device/1', 4, 0.5)"
            % os.path.join(ROOT, "spectral-kernel-benchmarks_b200"))
    env = dict(os.environ, SKB_TUNE_CACHE=str(path))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "32"
    assert path.read_text().splitlines() == ["32 1.5 stage A | test-device/1", "4 0.5 stage B | test-device/1"]
