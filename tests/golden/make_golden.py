"""Generate the golden fixtures in this folder from the reference's own code.

Run in a container where the reference tree exists (it is compiled in place by
``make -C oracle ref`` into oracle/_ref/libskbref.so):

    python tests/golden/make_golden.py

Every number written here comes from the reference's functions
(src/model.cpp, src/pointwise_advection.cpp, src/json.cpp,
src/spectral_flux_fixture.cpp) through the thin shim oracle/ref_shim.cpp
(the two-family fixture's inputs and matrices are seeded data; its expected
targets come from the reference's functions).  The fixtures are small (tens of KB) so that the
tests can pin the oracle restatement and the CUDA provider without the
reference tree, which is absent on the GPU host.
"""

import ctypes
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libskbref.so")

U64 = ctypes.c_uint64


def p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def load():
    ref = os.environ.get("REF", "/root/reference")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "REF=" + ref], check=True)
    lib = ctypes.CDLL(REF_LIB)
    lib.skbref_last_error.restype = ctypes.c_char_p
    lib.skbref_max_rel_error_complex.restype = ctypes.c_double
    lib.skbref_rel_l2_error.restype = ctypes.c_double
    return lib


def check(lib, rc):
    if rc != 0:
        raise RuntimeError(lib.skbref_last_error().decode())


def modes(lib, n, nz, fields):
    H = n * (n // 2 + 1)
    k = np.zeros(H, np.int64)
    l = np.zeros(H, np.int64)
    kx = np.zeros(H, np.uint64)
    ky = np.zeros(H, np.uint64)
    c = np.zeros(H, np.uint8)
    r = np.zeros(H)
    cnt = U64()
    check(lib, lib.skbref_retained_modes(U64(n), U64(n), U64(nz), U64(fields), p(k), p(l), p(kx), p(ky), p(c), p(r),
                                         ctypes.byref(cnt)))
    m = cnt.value
    return dict(k=k[:m], l=l[:m], kx=kx[:m].astype(np.int64), ky=ky[:m].astype(np.int64), conj=c[:m], radial=r[:m])


def groups(lib, n, nz, fields):
    H = n * (n // 2 + 1)
    keys = np.zeros(H, np.uint64)
    first = np.zeros(H, np.uint64)
    counts = np.zeros(H, np.uint64)
    g = U64()
    bufs = [ctypes.create_string_buffer(64) for _ in range(3)]
    check(lib, lib.skbref_groups_and_hashes(U64(n), U64(n), U64(nz), U64(fields), p(keys), p(first), p(counts),
                                            ctypes.byref(g), *bufs))
    m = g.value
    return keys[:m], first[:m].astype(np.int64), counts[:m].astype(np.int64), [b.value.decode() for b in bufs]


def fixture(lib, n, nz, fields, kind, seed):
    out = np.zeros(n * n * nz * fields)
    check(lib, lib.skbref_make_fixture(U64(n), U64(n), U64(nz), U64(fields), ctypes.c_int(kind), U64(seed), p(out)))
    return out


def direct_r2c(lib, n, nz, fields, real):
    out = np.zeros(2 * n * (n // 2 + 1) * nz * fields)
    check(lib, lib.skbref_direct_r2c(U64(n), U64(n), U64(nz), U64(fields), p(real), p(out)))
    return out.view(np.complex128)


def direct_c2r(lib, n, nz, fields, spec):
    out = np.zeros(n * n * nz * fields)
    s = np.ascontiguousarray(spec).view(np.float64)
    check(lib, lib.skbref_direct_c2r(U64(n), U64(n), U64(nz), U64(fields), p(s), p(out)))
    return out


def two_family_fixture(lib, n=16, nz=7, seed=11):
    """The authoritative two-family flux, pinned to the reference: a synthetic
    prepared fixture (SKFXP001; seeded floating K^2 groups, wave-f / wave-g
    matrices, modal inputs, modes stored in the file in reverse order within each
    group) is written, read by the reference's own loader
    (loadPreparedSpectralFluxFixture), and its expected targets are the flux that
    oracle/ref_shim.cpp composes from the reference's functions with the
    fixture's family maps.  The file (with those targets) is kept beside this
    script as two_family_16x7.skfxp; the loader's view of it goes into the
    returned arrays (two_family_*)."""
    for path in (ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "spectral-kernel-benchmarks_b200")):
        if path not in sys.path:
            sys.path.insert(0, path)
    import skb_cuda.fixture as fx
    from synthetic_fixture import families_canonical

    modes, fam, group_keys = families_canonical(n, nz, seed)
    H = len(modes.k)
    nj = 2 * (nz - 1) // 3
    rng = np.random.default_rng(seed + 1)
    inputs = rng.uniform(-0.125, 0.125, (H, 15, nj)) + 1j * rng.uniform(-0.125, 0.125, (H, 15, nj))
    inputs[0].imag = 0.0
    counts = fam["group_modes"].astype(np.int64)
    first = np.r_[0, np.cumsum(counts)[:-1]]
    order = np.concatenate([np.arange(f0 + c - 1, f0 - 1, -1) for f0, c in zip(first, counts)])
    group_of = np.repeat(np.arange(len(counts)), counts)
    keys = np.stack([modes.k, modes.l], axis=1)
    path = os.path.join(HERE, "two_family_16x7.skfxp")
    meta = {"fixture_id": "synthetic-two-family-16x7", "generator": "tests/golden/make_golden.py"}

    def write(targets):
        fx.write(path, n, nz, keys[order], group_of, group_keys, fam["forward"], fam["inverse"], inputs[order],
                 targets[order], meta=meta)

    write(np.zeros((H, 4, nj), np.complex128))
    targets = np.zeros(2 * H * 4 * nj)
    check(lib, lib.skbref_two_family_flux_direct(path.encode(), p(targets)))
    targets = targets.view(np.complex128).reshape(H, 4, nj)
    write(targets)

    dims = np.zeros(6, np.uint64)
    check(lib, lib.skbref_load_flux_fixture(path.encode(), p(dims), *([None] * 10)))
    _, _, nkl, nj2, ngroups, nsource = (int(v) for v in dims)
    k = np.zeros(nkl, np.int64)
    l = np.zeros(nkl, np.int64)
    gfirst, gcount, gkey, gsource = (np.zeros(ngroups, np.uint64) for _ in range(4))
    fwd = np.zeros(2 * nsource * nj2 * nz)
    inv = np.zeros(2 * nsource * nj2 * nz)
    modal_in = np.zeros(2 * nkl * 15 * nj2)
    expected = np.zeros(2 * nkl * 4 * nj2)
    check(lib, lib.skbref_load_flux_fixture(path.encode(), p(dims), p(k), p(l), p(gfirst), p(gcount), p(gkey),
                                            p(gsource), p(fwd), p(inv), p(modal_in), p(expected)))
    return {"two_family_k": k, "two_family_l": l, "two_family_group_first": gfirst,
            "two_family_group_count": gcount, "two_family_group_key": gkey, "two_family_matrix_source": gsource,
            "two_family_forward": fwd.reshape(2, nsource, nj2, nz), "two_family_inverse": inv.reshape(2, nsource, nz, nj2),
            "two_family_inputs": modal_in.view(np.complex128).reshape(nkl, 15, nj2),
            "two_family_targets": expected.view(np.complex128).reshape(nkl, 4, nj2)}


def main():
    lib = load()
    golden = {}

    # Known answers: counts and order hashes for every profile class the path uses.
    sizes = [(8, 7, 2), (16, 7, 2), (32, 9, 3), (64, 17, 3), (128, 33, 3), (256, 65, 3), (256, 129, 4),
             (512, 129, 4), (1024, 129, 4)]
    known = []
    for n, nz, f in sizes:
        m = modes(lib, n, nz, f)
        keys, first, counts, (mh, gh, wh) = groups(lib, n, nz, f)
        known.append(dict(n=n, nz=nz, fields=f, modes=int(len(m["k"])), groups=int(len(keys)), mode_hash=mh,
                          group_hash=gh, wvm_hash=wh, active_kx=int(m["kx"].max()) + 1,
                          max_group=int(counts.max())))
    golden["known_answers"] = known

    # Full-size fixture generator checksums (makeFixture, model.cpp:618-661).
    sums = []
    for n, nz, f, kind, seed in [(256, 65, 3, 2, 129), (64, 9, 2, 1, 130), (64, 9, 2, 0, 129), (64, 9, 2, 4, 133)]:
        v = fixture(lib, n, nz, f, kind, seed)
        sums.append(dict(n=n, nz=nz, fields=f, kind=kind, seed=seed, sha256=hashlib.sha256(v.tobytes()).hexdigest()))
    golden["fixture_sha256"] = sums

    with open(os.path.join(HERE, "known_answers.json"), "w") as fh:
        json.dump(golden, fh, indent=1)

    # validate --profile smoke (benchmark.cpp:4898-5003): 8x8x7x2, fixtures 0..4, seeds 129+i.
    n, nz, f = 8, 7, 2
    arrays = {}
    m = modes(lib, n, nz, f)
    for key, val in m.items():
        arrays["smoke_modes_" + key] = val
    nj = 2 * (nz - 1) // 3
    fwd = np.zeros(nj * nz)
    inv = np.zeros(nj * nz)
    check(lib, lib.skbref_orthonormal_vertical_fixture(U64(nz), U64(nj), p(fwd), p(inv)))
    arrays["smoke_vertical_forward"] = fwd
    arrays["smoke_vertical_inverse"] = inv
    for i in range(5):
        real = fixture(lib, n, nz, f, i, 129 + i)
        spec = direct_r2c(lib, n, nz, f, real)
        ret = np.zeros(2 * len(m["k"]) * nz * f)
        check(lib, lib.skbref_gather_retained(U64(n), U64(n), U64(nz), U64(f), p(spec.view(np.float64)), p(ret)))
        emb = np.zeros(2 * n * (n // 2 + 1) * nz * f)
        check(lib, lib.skbref_embed_retained(U64(n), U64(n), U64(nz), U64(f), p(ret), p(emb)))
        back = direct_c2r(lib, n, nz, f, spec)
        arrays[f"smoke_{i}_real"] = real
        arrays[f"smoke_{i}_spectrum"] = spec
        arrays[f"smoke_{i}_retained"] = ret.view(np.complex128)
        arrays[f"smoke_{i}_embedded"] = emb.view(np.complex128)
        arrays[f"smoke_{i}_c2r"] = back

    # A larger direct-DFT case (32x32, 3 planes x 2 fields) for the full FFT and the pruned path.
    n, nz, f = 32, 3, 2
    real = fixture(lib, n, nz, f, 2, 700)
    spec = direct_r2c(lib, n, nz, f, real)
    arrays["d32_real"] = real
    arrays["d32_spectrum"] = spec
    arrays["d32_c2r"] = direct_c2r(lib, n, nz, f, spec)
    m32 = modes(lib, n, nz, f)
    ret = np.zeros(2 * len(m32["k"]) * nz * f)
    check(lib, lib.skbref_gather_retained(U64(n), U64(n), U64(nz), U64(f), p(spec.view(np.float64)), p(ret)))
    arrays["d32_retained"] = ret.view(np.complex128)
    emb = np.zeros(2 * n * (n // 2 + 1) * nz * f)
    check(lib, lib.skbref_embed_retained(U64(n), U64(n), U64(nz), U64(f), p(ret), p(emb)))
    arrays["d32_embedded_c2r"] = direct_c2r(lib, n, nz, f, emb.view(np.complex128))

    # K^2 vertical family and grouped projections at 16x16, Nz=9, 3 fields.
    n, nz, f = 16, 9, 3
    keys, first, counts, _ = groups(lib, n, nz, f)
    nj = 2 * (nz - 1) // 3
    G = len(keys)
    fam_f = np.zeros(G * nj * nz)
    fam_i = np.zeros(G * nj * nz)
    njo = U64()
    ident = ctypes.create_string_buffer(128)
    check(lib, lib.skbref_k2_vertical_fixture(U64(n), U64(n), U64(nz), U64(f), p(fam_f), p(fam_i), ctypes.byref(njo),
                                              ident))
    H = int(first[-1] + counts[-1])
    rng = np.random.default_rng(5)
    phys = (rng.uniform(-1, 1, H * f * nz) + 1j * rng.uniform(-1, 1, H * f * nz)).astype(np.complex128)
    modal = np.zeros(2 * H * f * nj)
    check(lib, lib.skbref_grouped_vertical(U64(n), U64(n), U64(nz), U64(f), ctypes.c_int(0), p(phys.view(np.float64)),
                                           p(modal)))
    modal_in = (rng.uniform(-1, 1, H * f * nj) + 1j * rng.uniform(-1, 1, H * f * nj)).astype(np.complex128)
    phys_out = np.zeros(2 * H * f * nz)
    check(lib, lib.skbref_grouped_vertical(U64(n), U64(n), U64(nz), U64(f), ctypes.c_int(1),
                                           p(modal_in.view(np.float64)), p(phys_out)))
    arrays.update(k2_keys=keys, k2_forward=fam_f, k2_inverse=fam_i, k2_phys=phys, k2_modal=modal.view(np.complex128),
                  k2_modal_in=modal_in, k2_phys_out=phys_out.view(np.complex128))
    golden_id = ident.value.decode()

    # Pointwise executor (tests/skbench_tests.cpp:1136-1185 inputs), all three policies.
    volume, scale = 37, 0.03125
    idx = np.arange(3 * volume)
    shared = (idx % 17 - 8.0).astype(np.float64)
    deriv = ((3 * idx + 5) % 23 - 11.0).astype(np.float64)
    for policy, workers in [(0, 1), (1, 1), (2, 4)]:
        out = np.zeros(volume)
        check(lib, lib.skbref_pointwise(ctypes.c_int(policy), U64(workers), U64(volume), ctypes.c_double(scale),
                                        p(shared), p(deriv), p(out)))
        arrays[f"pointwise_{policy}"] = out
    arrays["pointwise_shared"] = shared
    arrays["pointwise_derivative"] = deriv

    # The 15 -> 4 flux composed from the reference's functions, two small sizes.
    for n, nz in [(16, 7), (16, 13)]:
        m = modes(lib, n, nz, 4)
        nj = 2 * (nz - 1) // 3
        H = len(m["k"])
        mi = np.zeros(2 * H * 15 * nj)
        mo = np.zeros(2 * H * 4 * nj)
        check(lib, lib.skbref_flux_direct(U64(n), U64(nz), U64(129), p(mi), p(mo)))
        arrays[f"flux{n}_{nz}_in"] = mi.view(np.complex128)
        arrays[f"flux{n}_{nz}_out"] = mo.view(np.complex128)

    # The spectral-pipeline round trip composed from the reference's functions.
    n, nz, f = 16, 9, 2
    m = modes(lib, n, nz, f)
    nj = 2 * (nz - 1) // 3
    pin = np.zeros(n * n * nz * f)
    pw = np.zeros(len(m["k"]) * f * nj)
    pout = np.zeros(n * n * nz * f)
    check(lib, lib.skbref_spectral_pipeline(U64(n), U64(nz), U64(f), U64(129), p(pin), p(pw), p(pout)))
    arrays.update(pipeline_in=pin, pipeline_weights=pw, pipeline_out=pout)

    arrays.update(two_family_fixture(lib))

    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **arrays)

    # The reference report writer's own output, for schema key comparison.
    check(lib, lib.skbref_write_schema_sample(os.path.join(HERE, "reference_report.json").encode(),
                                              os.path.join(HERE, "reference_report.csv").encode()))
    with open(os.path.join(HERE, "known_answers.json")) as fh:
        golden = json.load(fh)
    golden["k2_family_id"] = golden_id
    with open(os.path.join(HERE, "known_answers.json"), "w") as fh:
        json.dump(golden, fh, indent=1)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    sys.exit(main())
