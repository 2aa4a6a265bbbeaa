"""ORACLE — test infrastructure only.

CPU restatement of the reference (JeffreyEarly/spectral-kernel-benchmarks)
arithmetic on the spectral hot path.  Only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs import this module, and only as the
checker or the timed CPU baseline: the CUDA provider never calls it.

Small exact pieces (retained modes, K^2 groups, FNV order hashes, fixtures with
the mt19937_64 + normal_distribution generator, the O(N^4) direct DFTs) live in
oracle/skb_oracle.cpp (liboracle.so).  Full-size transforms use numpy's
pocketfft in float64, mapped to the reference's WVM frequency-major layout;
they are pinned to the direct DFT by tests/test_oracle_pins.py.

Layouts (all follow include/skbench/skbench.hpp and src/model.cpp:219-244):
  real        [field][z][y][x]                      (x fastest)
  wvm         [ky][kx][field][z]                    (plane = z + nz*field fastest)
  retained    [mode][field][z]                      (z fastest)
  modal       [mode][field][j]                      (j fastest)
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def library():
    """Load liboracle.so, building it with the oracle Makefile when absent."""
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
        lib = ctypes.CDLL(path)
        lib.oracle_last_error.restype = ctypes.c_char_p
        _LIB = lib
    return _LIB


def _p(array):
    return array.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError(library().oracle_last_error().decode())


U64 = ctypes.c_uint64


@dataclass(frozen=True)
class Workload:
    """skbench.hpp:23-39 Workload; lx = ly = 1 and antialias on, as every profile."""
    nx: int
    ny: int
    nz: int
    fields: int

    @property
    def planes(self):
        return self.nz * self.fields

    @property
    def nx_half(self):
        return self.nx // 2 + 1

    @property
    def nj(self):
        """model.cpp:124-127: floor(2*(Nz-1)/3)."""
        return 0 if self.nz < 2 else 2 * (self.nz - 1) // 3


@dataclass
class Modes:
    k: np.ndarray
    l: np.ndarray
    kx: np.ndarray
    ky: np.ndarray
    conj: np.ndarray
    radial: np.ndarray

    def __len__(self):
        return len(self.k)


def retained_modes(nx, ny):
    """model.cpp:129-167 radial 2/3 retained modes (see skb_oracle.cpp)."""
    cap = nx * (nx // 2 + 1) + ny
    k = np.zeros(cap, np.int64)
    l = np.zeros(cap, np.int64)
    kx = np.zeros(cap, np.uint64)
    ky = np.zeros(cap, np.uint64)
    conj = np.zeros(cap, np.uint8)
    radial = np.zeros(cap)
    count = U64()
    _check(library().oracle_retained_modes(U64(nx), U64(ny), ctypes.c_double(1.0), ctypes.c_double(1.0),
                                           ctypes.c_int(1), _p(k), _p(l), _p(kx), _p(ky), _p(conj), _p(radial),
                                           U64(cap), ctypes.byref(count)))
    n = count.value
    return Modes(k[:n].copy(), l[:n].copy(), kx[:n].astype(np.int64), ky[:n].astype(np.int64),
                 conj[:n].astype(bool), radial[:n].copy())


def k2_groups(nx, ny):
    """model.cpp:169-207: (keys, first, counts) of the contiguous K^2 groups."""
    cap = nx * (nx // 2 + 1) + ny
    keys = np.zeros(cap, np.uint64)
    first = np.zeros(cap, np.uint64)
    counts = np.zeros(cap, np.uint64)
    count = U64()
    _check(library().oracle_groups(U64(nx), U64(ny), _p(keys), _p(first), _p(counts), U64(cap), ctypes.byref(count)))
    n = count.value
    return keys[:n].copy(), first[:n].astype(np.int64), counts[:n].astype(np.int64)


def hashes(w: Workload):
    """(retained mode order, K^2 group order, WVM full-spectrum order) FNV-1a hashes."""
    bufs = [ctypes.create_string_buffer(64) for _ in range(3)]
    _check(library().oracle_hashes(U64(w.nx), U64(w.ny), U64(w.nz), U64(w.fields), *bufs))
    return tuple(b.value.decode() for b in bufs)


FIXTURES = ("impulse", "sinusoid", "random", "dc", "nyquist")


def make_fixture(w: Workload, kind, seed):
    """model.cpp:618-661 makeFixture -> real[field][z][y][x]."""
    kind_index = FIXTURES.index(kind) if isinstance(kind, str) else int(kind)
    out = np.zeros(w.nx * w.ny * w.planes)
    _check(library().oracle_make_fixture(U64(w.nx), U64(w.ny), U64(w.nz), U64(w.fields), ctypes.c_int(kind_index),
                                         U64(seed), _p(out)))
    return out


def flux_inputs(modes: Modes, fields, nj, seed):
    """benchmark.cpp:4045-4058 modal inputs [mode][field][j] (complex128)."""
    out = np.zeros(2 * len(modes) * fields * nj)
    k = np.ascontiguousarray(modes.k)
    l = np.ascontiguousarray(modes.l)
    _check(library().oracle_flux_inputs(_p(k), _p(l), U64(len(modes)), U64(fields), U64(nj), U64(seed), _p(out)))
    return out.view(np.complex128)


def direct_r2c(w: Workload, real):
    """model.cpp:663-684 direct DFT -> WVM spectrum (complex128, flat)."""
    out = np.zeros(2 * w.ny * w.nx_half * w.planes)
    real = np.ascontiguousarray(real, dtype=np.float64)
    _check(library().oracle_direct_r2c(U64(w.nx), U64(w.ny), U64(w.planes), _p(real), _p(out)))
    return out.view(np.complex128)


def direct_c2r(w: Workload, wvm):
    """model.cpp:686-716 direct inverse DFT (unnormalised) -> real."""
    out = np.zeros(w.nx * w.ny * w.planes)
    spec = np.ascontiguousarray(wvm, dtype=np.complex128).view(np.float64)
    _check(library().oracle_direct_c2r(U64(w.nx), U64(w.ny), U64(w.planes), _p(spec), _p(out)))
    return out


def fft_r2c(w: Workload, real, workers=1):
    """FFTWProvider::forward (fftw_provider.cpp:537-572) restated with pocketfft:
    unnormalised 2-D r2c of every plane, written frequency-major (WVM).
    workers > 1 uses scipy.fft's threaded pocketfft (timing baselines)."""
    planes = np.asarray(real, dtype=np.float64).reshape(w.planes, w.ny, w.nx)
    if workers > 1:
        import scipy.fft

        spec = scipy.fft.rfft2(planes, axes=(1, 2), workers=workers)
    else:
        spec = np.fft.rfft2(planes, axes=(1, 2))  # [plane][ky][kx]
    return np.ascontiguousarray(spec.transpose(1, 2, 0)).reshape(-1)


def fft_c2r(w: Workload, wvm, workers=1):
    """FFTWProvider::inverse (fftw_provider.cpp:574-610): unnormalised c2r with
    FFTW's half-spectrum semantics (columns c2c, then rows c2r; the imaginary
    parts of the kx = 0 and kx = Nx/2 bins of each row are ignored)."""
    spec = np.asarray(wvm, dtype=np.complex128).reshape(w.ny, w.nx_half, w.planes).transpose(2, 0, 1)
    if workers > 1:
        import scipy.fft

        real = scipy.fft.irfft2(spec, s=(w.ny, w.nx), axes=(1, 2), norm="forward", workers=workers)
    else:
        real = np.fft.irfft2(spec, s=(w.ny, w.nx), axes=(1, 2), norm="forward")
    return np.ascontiguousarray(real).reshape(-1)


def gather_retained(w: Workload, modes: Modes, wvm, scale=1.0):
    """model.cpp:310-321 gatherRetained -> retained [mode][plane]."""
    spec = np.asarray(wvm).reshape(w.ny, w.nx_half, w.planes)
    vals = spec[modes.ky, modes.kx, :]
    vals = np.where(modes.conj[:, None], np.conj(vals), vals)
    return (scale * vals).reshape(-1)


def embed_retained(w: Workload, modes: Modes, retained):
    """model.cpp:323-339 embedRetained: zero-fill, scatter, kx = 0 Hermitian partner."""
    comp = np.asarray(retained).reshape(len(modes), w.planes)
    stored = np.where(modes.conj[:, None], np.conj(comp), comp)
    spec = np.zeros((w.ny, w.nx_half, w.planes), np.complex128)
    spec[modes.ky, modes.kx, :] = stored
    rep = (modes.kx == 0) & (modes.ky != 0) & (2 * modes.ky != w.ny)
    spec[(w.ny - modes.ky[rep]) % w.ny, 0, :] = np.conj(stored[rep])
    return spec.reshape(-1)


def k2_family(w: Workload):
    """model.cpp:523-565 squaredWavenumberVerticalFixture: (forward[g][j][z], inverse[g][z][j])."""
    keys, _, _ = k2_groups(w.nx, w.ny)
    nj, nz = w.nj, w.nz
    fwd = np.zeros(len(keys) * nj * nz)
    inv = np.zeros(len(keys) * nj * nz)
    keys = np.ascontiguousarray(keys)
    _check(library().oracle_k2_vertical_family(U64(nz), U64(nj), _p(keys), U64(len(keys)), _p(fwd), _p(inv)))
    return fwd.reshape(len(keys), nj, nz), inv.reshape(len(keys), nz, nj)


def sturm_liouville_family(w: Workload, seed):
    """The build-side seeded Sturm-Liouville vertical family (the perf-realistic
    dense operators; the reference has none): per K^2 group, the lowest Nj
    eigenvectors of the tridiagonal discretisation of -d/dz (1/N^2 d/dz) + 1e-3
    K^2/N^2 on a unit-depth grid of Nz cells with Neumann ends, where
    1/N^2 = exp(-(z_i - 1)/h) at cell interfaces z_i = i/Nz and h is the seeded
    scale height.  Eigenvectors from LAPACK (scipy eigh_tridiagonal), ordered
    by eigenvalue, signed so their first entry above 1e-12 in magnitude is
    positive.  Returns (forward[g][j][z], inverse[g][z][j])."""
    from scipy.linalg import eigh_tridiagonal

    h = ctypes.c_double()
    _check(library().oracle_sl_scale_height(U64(seed), ctypes.byref(h)))
    keys, _, _ = k2_groups(w.nx, w.ny)
    nz, nj = w.nz, w.nj
    dz = 1.0 / nz
    inv = np.exp(-(np.arange(nz + 1) * dz - 1.0) / h.value)
    up = np.where(np.arange(nz) + 1 < nz, inv[1:], 0.0)
    dn = np.where(np.arange(nz) > 0, inv[:-1], 0.0)
    base = (up + dn) / (dz * dz)
    mid = 0.5 * (inv[:-1] + inv[1:])
    off = -inv[1:nz] / (dz * dz)
    fwd = np.empty((len(keys), nj, nz))
    for g, key in enumerate(keys):
        k2 = 4.0 * np.pi * np.pi * float(key)
        vals, vecs = eigh_tridiagonal(base + 1e-3 * k2 * mid, off)
        vecs = vecs[:, np.argsort(vals, kind="stable")[:nj]].T
        for j in range(nj):
            first = np.flatnonzero(np.abs(vecs[j]) > 1e-12)
            if first.size and vecs[j, first[0]] < 0:
                vecs[j] = -vecs[j]
        fwd[g] = vecs
    return fwd, np.ascontiguousarray(fwd.transpose(0, 2, 1))


def grouped_vertical(w: Workload, family, direction, data):
    """Per-group vertical projection (model.cpp:567-605 applied per K^2 group, as
    VerticalGemmProvider does, vertical_gemm.cpp:534-596).  forward: retained
    [mode][field][z] -> modal [mode][field][j]; inverse the reverse."""
    fwd, inv = family
    _, first, counts = k2_groups(w.nx, w.ny)
    rows_in, rows_out, mats = (w.nz, w.nj, fwd) if direction == "forward" else (w.nj, w.nz, inv)
    H = int(first[-1] + counts[-1])
    x = np.asarray(data, dtype=np.complex128).reshape(H * w.fields, rows_in)
    out = np.empty((H * w.fields, rows_out), np.complex128)
    for g, (f0, c) in enumerate(zip(first, counts)):
        a, b = f0 * w.fields, (f0 + c) * w.fields
        out[a:b] = x[a:b] @ mats[g].T
    return out.reshape(-1)


def pointwise(volume, scale, shared, derivative, workers=1):
    """pointwise_advection.cpp:143-147: -scale*(u*qx + v*qy + w*qz)."""
    shared = np.ascontiguousarray(shared, dtype=np.float64)
    derivative = np.ascontiguousarray(derivative, dtype=np.float64)
    out = np.empty(volume)
    _check(library().oracle_pointwise(U64(volume), ctypes.c_double(scale), _p(shared), _p(derivative), _p(out),
                                      U64(workers)))
    return out


def family_vertical(families, direction, data, fields, rows_in, rows_out, field_family):
    """Per operator group and field, the field's family matrix (the
    authoritative WVM form: VerticalGemmProvider calls partitioned by family,
    authoritative_spectral_flux.cpp:1409-1571).  families: 'group_modes',
    'forward' / 'inverse' per family [group][j][z] / [group][z][j]."""
    counts = np.asarray(families["group_modes"], np.int64)
    first = np.r_[0, np.cumsum(counts)[:-1]]
    H = int(counts.sum())
    mats = families["forward" if direction == "forward" else "inverse"]
    x = np.asarray(data, dtype=np.complex128).reshape(H, fields, rows_in)
    out = np.empty((H, fields, rows_out), np.complex128)
    for g, (f0, c) in enumerate(zip(first, counts)):
        for f in range(fields):
            out[f0:f0 + c, f] = x[f0:f0 + c, f] @ np.asarray(mats[field_family[f]][g]).T
    return out.reshape(-1)


def flux(n, nz, modal_in, targets=4, family=None, modes=None, workers=1, families=None):
    """The 15 -> 4 streamed flux of runProductionLifetimeFluxBenchmark
    (benchmark.cpp:4182-4241 oracle order, 4405-4424 executeAll): inverse
    vertical GEMM of all input fields, inverse horizontal of [U,V,W] once, then per
    target the inverse of its derivative triple, pointwise advection with
    scale 1/(Nx*Ny)^2, forward horizontal + retention, and finally the forward
    vertical GEMM of the targets.  ``targets`` = 3 gives the 12 -> 3 variant;
    ``families`` (see family_vertical) gives the authoritative two-family form.
    Returns modal [mode][target][j]."""
    fields_in = 3 + 3 * targets
    w_in = Workload(n, n, nz, fields_in)
    w_out = Workload(n, n, nz, targets)
    w3 = Workload(n, n, nz, 3)
    w1 = Workload(n, n, nz, 1)
    modes = modes or retained_modes(n, n)
    H = len(modes)
    if families is not None:
        phys = family_vertical(families, "inverse", modal_in, fields_in, w_in.nj, nz,
                               families["input_family"]).reshape(H, fields_in, nz)
    else:
        family = family or k2_family(w_out)
        phys = grouped_vertical(w_in, family, "inverse", modal_in).reshape(H, fields_in, nz)
    scale = 1.0 / float((n * n) ** 2)
    shared = fft_c2r(w3, embed_retained(w3, modes, phys[:, 0:3, :].reshape(-1)), workers)
    phys_out = np.empty((H, targets, nz), np.complex128)
    for t in range(targets):
        trip = phys[:, 3 + 3 * t:6 + 3 * t, :].reshape(-1)
        deriv = fft_c2r(w3, embed_retained(w3, modes, trip), workers)
        target = pointwise(n * n * nz, scale, shared, deriv, workers)
        phys_out[:, t, :] = gather_retained(w1, modes, fft_r2c(w1, target, workers)).reshape(H, nz)
    if families is not None:
        return family_vertical(families, "forward", phys_out.reshape(-1), targets, nz, w_out.nj,
                               families["target_family"])
    return grouped_vertical(w_out, family, "forward", phys_out.reshape(-1))


def max_rel_error(actual, expected):
    """model.cpp:718-726: max |a-b| / max(1, max |b|)."""
    a = np.asarray(actual).reshape(-1)
    b = np.asarray(expected).reshape(-1)
    return float(np.max(np.abs(a - b), initial=0.0) / max(1.0, float(np.max(np.abs(b), initial=0.0))))


def rel_l2_error(actual, expected):
    """model.cpp:738-751: ||a-b||_2 / ||b||_2 (absolute when ||b|| = 0)."""
    a = np.asarray(actual, dtype=np.complex128).reshape(-1)
    b = np.asarray(expected, dtype=np.complex128).reshape(-1)
    num = float(np.sum(np.abs(a - b) ** 2))
    den = float(np.sum(np.abs(b) ** 2))
    return float(np.sqrt(num if den == 0.0 else num / den))


def wvm_direct_vertical(w: Workload, family, direction, data, out=None):
    """WvmDirectVerticalGemmProvider::executeForward / executeInverse
    (vertical_gemm.cpp:935-1169): per retained mode, the group's real matrix
    times the mode's stored WVM cell, fields as columns, no conjugation
    (forwardMode / inverseMode), then the kx = 0 boundary copy: the partner
    cell (0, Ny - ky) receives the conjugate (copyModalBoundary /
    copySpectrumBoundary).  forward: WVM spectrum [ky][kx][field][z] -> WVM modal
    spectrum [ky][kx][field][j]; inverse the reverse.  Cells of `out` that are
    not written keep their values (the provider's initialize*Output zero them)."""
    fwd, inv = family
    modes = retained_modes(w.nx, w.ny)
    _, first, counts = k2_groups(w.nx, w.ny)
    group_of = np.repeat(np.arange(len(first)), counts)
    half = w.nx // 2 + 1
    rows_in, rows_out, mats = (w.nz, w.nj, fwd) if direction == "forward" else (w.nj, w.nz, inv)
    x = np.asarray(data, dtype=np.complex128).reshape(w.ny, half, w.fields, rows_in)
    y = np.zeros((w.ny, half, w.fields, rows_out), np.complex128) if out is None else \
        np.array(out, dtype=np.complex128).reshape(w.ny, half, w.fields, rows_out)
    for m in range(len(modes)):
        kx, ky = int(modes.kx[m]), int(modes.ky[m])
        y[ky, kx] = x[ky, kx] @ mats[group_of[m]].T
    for m in range(len(modes)):
        kx, ky = int(modes.kx[m]), int(modes.ky[m])
        if kx == 0 and ky != 0 and 2 * ky != w.ny:
            y[(w.ny - ky) % w.ny, 0] = np.conj(y[ky, 0])
    return y.reshape(-1)


def modal_weights(w: Workload):
    """syntheticModalWorkWeights (model.cpp:246-267): per (mode, field, j),
    0.75 + 0.5 * ((17|k| + 29|l| + 7j + 11 field) mod 97) / 96, [mode][field][j]."""
    modes = retained_modes(w.nx, w.ny)
    k = np.abs(np.asarray(modes.k, np.int64))
    l = np.abs(np.asarray(modes.l, np.int64))
    f = np.arange(w.fields)[None, :, None]
    j = np.arange(w.nj)[None, None, :]
    key = (17 * k[:, None, None] + 29 * l[:, None, None] + 7 * j + 11 * f) % 97
    return (0.75 + 0.5 * key / 96.0).reshape(-1)


def spectral_pipeline(w: Workload, real, family=None, workers=1):
    """The spectral-pipeline round trip (benchmark.cpp:3072-3110 reference order):
    r2c, retention, K^2 vertical forward, synthetic modal work, vertical inverse,
    embedding, c2r (unnormalised, FFTW semantics)."""
    family = k2_family(w) if family is None else family
    modes = retained_modes(w.nx, w.ny)
    spec = fft_r2c(w, real, workers)
    ret = gather_retained(w, modes, spec)
    modal = grouped_vertical(w, family, "forward", ret) * modal_weights(w)
    back = grouped_vertical(w, family, "inverse", modal)
    return fft_c2r(w, embed_retained(w, modes, back), workers)


# ------------------------------------------------ constant stratification
# Type-I vertical transforms of the constant-stratification kernel
# (src/constant_stratification.cpp).  Arrays are complex [row][channel][z]
# (index(), 154-157).  The transforms are the FFTW r2r kinds the reference
# plans (R2RPlan, 95-146): REDFT00 over all nz points and RODFT00 over the
# nz-2 interior points, applied to the real and imaginary parts alike.  Here
# they are direct sums with cosine / sine tables indexed by (k z mod 2(nz-1)),
# so every table entry is an exactly reduced angle.

def _type1_tables(nz):
    m = nz - 1
    kz = (np.arange(nz)[:, None] * np.arange(nz)[None, :]) % (2 * m)
    angle = np.pi * kz.astype(np.float64) / m
    return np.cos(angle), np.sin(angle)


def dct1(column):
    """REDFT00 along the last axis: Y_k = x_0 + (-1)^k x_{nz-1}
    + 2 sum_{z=1}^{nz-2} x_z cos(pi k z / (nz-1))."""
    x = np.asarray(column, dtype=np.complex128)
    nz = x.shape[-1]
    c, _ = _type1_tables(nz)
    w = 2.0 * c
    w[:, 0] = 1.0
    w[:, nz - 1] = np.where(np.arange(nz) % 2 == 0, 1.0, -1.0)
    return x @ w.T


def dst1_interior(column):
    """RODFT00 on the interior z = 1 .. nz-2 (endpoints returned unchanged):
    Y_k = 2 sum_{z=1}^{nz-2} x_z sin(pi k z / (nz-1))."""
    x = np.asarray(column, dtype=np.complex128)
    nz = x.shape[-1]
    _, s = _type1_tables(nz)
    w = 2.0 * s[1:nz - 1, 1:nz - 1]
    out = x.copy()
    out[..., 1:nz - 1] = x[..., 1:nz - 1] @ w.T
    return out


def normalize_dct1(column):
    """normalizeForwardDct (constant_stratification.cpp:199-212): every value
    times 1/(nz-1), then the last one times 0.5."""
    y = np.array(column, dtype=np.complex128)
    nz = y.shape[-1]
    y *= 1.0 / float(nz - 1)
    y[..., nz - 1] *= 0.5
    return y


def normalize_dst1(column):
    """normalizeForwardDst (214-231): endpoints zero, interior times 1/(nz-1)."""
    y = np.array(column, dtype=np.complex128)
    nz = y.shape[-1]
    y[..., 1:nz - 1] *= 1.0 / float(nz - 1)
    y[..., 0] = 0.0
    y[..., nz - 1] = 0.0
    return y


def type1_transform(data, kind, storage_channels, first, channels, normalize=False):
    """R2RPlan::execute (+ normalisation) on [row][storage_channels][nz];
    kind 'dct' or 'dst'."""
    a = np.array(data, dtype=np.complex128)
    if a.ndim != 3 or a.shape[1] != storage_channels:
        raise ValueError("type1_transform expects a [row][storage_channels][z] array")
    sel = a[:, first:first + channels, :]
    if kind == "dct":
        out = dct1(sel)
        if normalize:
            out = normalize_dct1(out)
    else:
        out = dst1_interior(sel)
        if normalize:
            out = normalize_dst1(out)
    a[:, first:first + channels, :] = out
    return a


def type1_schedule(arena3, arena1):
    """executeCompleteVerticalGraph (constant_stratification.cpp:359-379):
    3 x (DCT-I on channels 0-1, DST-I on channel 2) and 2 x (DST-I on
    channels 0-1, DCT-I on channel 2) of the 3-channel arena, then 2 x
    normalised DCT-I and 2 x normalised DST-I of the 1-channel arena."""
    a3 = np.array(arena3, dtype=np.complex128)
    a1 = np.array(arena1, dtype=np.complex128)
    for _ in range(3):
        a3 = type1_transform(a3, "dct", 3, 0, 2)
        a3 = type1_transform(a3, "dst", 3, 2, 1)
    for _ in range(2):
        a3 = type1_transform(a3, "dst", 3, 0, 2)
        a3 = type1_transform(a3, "dct", 3, 2, 1)
    for _ in range(2):
        a1 = type1_transform(a1, "dct", 1, 0, 1, normalize=True)
    for _ in range(2):
        a1 = type1_transform(a1, "dst", 1, 0, 1, normalize=True)
    return a3, a1


def type1_deterministic(rows, channels, nz, row_ids=None, conj=None):
    """deterministicValue / fillFull / fillCompact (constant_stratification.cpp:
    233-260): value(row, channel, z) = (sin a, cos 1.7a) with a = 0.017(1 +
    row mod 97) + 0.113(1 + channel) + 0.071(1 + z).  row_ids maps each array
    row to the row the value is taken from (the mode's storedKx + nxHalf *
    storedKy for compact arrays); conj marks rows stored conjugated."""
    ids = np.arange(rows) if row_ids is None else np.asarray(row_ids, np.int64)
    a = (0.017 * (1 + ids % 97)[:, None, None] + 0.113 * (1 + np.arange(channels))[None, :, None]
         + 0.071 * (1 + np.arange(nz))[None, None, :])
    v = np.sin(a) + 1j * np.cos(1.7 * a)
    if conj is not None:
        v = np.where(np.asarray(conj, bool)[:, None, None], np.conj(v), v)
    return v
