"""Prepared spectral-flux fixtures (the authoritative WVM boundary).

A prepared fixture is one little-endian binary file, the format the
reference's loadPreparedSpectralFluxFixture reads
(src/spectral_flux_fixture.cpp:150-411; docs/wvm-spectral-flux-fixture-contract.md):

    magic "SKFXP001", u32 version 1, u32 byte-order marker 0x01020304,
    u32 authoritative flag 1, u32 reserved 0
    u64 Nx, Ny, Nz, Nkl, Nj, group count, family count (2), input count (15),
        target count (4)
    f64 Lx, Ly, Lz, latitude, pointwise scale (= 1 / (Nx Ny)^2)
    8 strings (u64 length + bytes): fixture id, WVM repository, WVM commit,
        generator identity, fixture hash ("sha256:" + 64 hex), normalization,
        mode mapping, derivative convention
    i32 [Nkl][2] horizontal mode keys (k, l), i32 [Nj] vertical keys (0..Nj-1)
    u32 [Nkl] operator group of each mode (nondecreasing), u64 [groups] group
        keys (k^2 + l^2, nondecreasing)
    u32 [15] input-slot families, u32 [4] target families (0 wave-f, 1 wave-g)
    per group, per family: f64 inverse matrix, element (z, j) at z + Nz j
    per group, per family: f64 forward matrix, element (j, z) at j + Nj z
    complex128 [Nkl][15][Nj] modal inputs, complex128 [Nkl][4][Nj] expected
        modal targets (modes in the file's order)

`load` checks what the reference checks before any timing and returns the
data in this library's order: modes as retainedHorizontalModes orders them,
operator groups as runs of modes that share a file group (one matrix pair per
run), matrices as forward[g][j][z] / inverse[g][z][j].  `write` produces the
format from data in the file's order (tests use it for synthetic fixtures).
"""

from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

MAGIC = b"SKFXP001"
VERSION = 1
BYTE_ORDER = 0x01020304
REPOSITORY = "JeffreyEarly/wave-vortex-model"
INPUT_FAMILIES = (0, 0, 1, 0, 0, 1, 0, 0, 1, 1, 1, 0, 1, 1, 0)
TARGET_FAMILIES = (0, 0, 1, 1)
STRINGS = ("fixture_id", "repository", "commit", "generator", "fixture_hash", "normalization", "mode_mapping",
           "derivative_convention")


class FixtureError(ValueError):
    """The file is not a valid prepared spectral-flux fixture."""


@dataclass
class PreparedFixture:
    nx: int
    ny: int
    nz: int
    nj: int
    lx: float
    ly: float
    lz: float
    latitude: float
    pointwise_scale: float
    meta: dict
    group_modes: np.ndarray     # modes per operator group, in retained-mode order
    group_keys: np.ndarray      # k^2 + l^2 of each operator group
    forward: list               # family f: [group][j][z]
    inverse: list               # family f: [group][z][j]
    input_family: tuple
    target_family: tuple
    modal_inputs: np.ndarray    # [mode][15][j], retained-mode order
    expected_targets: np.ndarray  # [mode][4][j]


class _Reader:
    def __init__(self, data):
        self.data = data
        self.at = 0

    def take(self, n, label):
        if self.at + n > len(self.data):
            raise FixtureError(f"prepared spectral-flux fixture is truncated at {label}")
        out = self.data[self.at:self.at + n]
        self.at += n
        return out

    def scalar(self, fmt, label):
        return struct.unpack("<" + fmt, self.take(struct.calcsize(fmt), label))[0]

    def array(self, dtype, count, label):
        dt = np.dtype(dtype).newbyteorder("<")
        return np.frombuffer(self.take(dt.itemsize * count, label), dtype=dt, count=count).copy()

    def string(self, label):
        n = self.scalar("Q", label)
        raw = self.take(n, label)
        if b"\0" in raw:
            raise FixtureError(f"{label} contains NUL bytes")
        return raw.decode("utf-8")


def _require(ok, message):
    if not ok:
        raise FixtureError(message)


def _retained_keys(nx, ny):
    import skb_cuda

    w = skb_cuda.Workload(nx, ny, 3, 1)
    return [(m.k, m.l) for m in skb_cuda.retained_modes(w)]


def load(path, retained_keys=None) -> PreparedFixture:
    """Read and validate a prepared fixture.  `retained_keys` (the (k, l) of
    retainedHorizontalModes, in order) defaults to the library's own."""
    with open(path, "rb") as fh:
        r = _Reader(fh.read())
    _require(r.take(8, "magic") == MAGIC, "prepared spectral-flux fixture has the wrong magic")
    _require(r.scalar("I", "version") == VERSION, "prepared spectral-flux fixture has an unsupported version")
    _require(r.scalar("I", "byte order") == BYTE_ORDER, "prepared spectral-flux fixture has the wrong byte order")
    _require(r.scalar("I", "authoritative flag") == 1, "prepared spectral-flux fixture is not authoritative")
    _require(r.scalar("I", "reserved word") == 0, "prepared spectral-flux fixture reserved header word is nonzero")
    nx, ny, nz, nkl, nj, ngroups, nfam, nin, nout = (r.scalar("Q", name) for name in (
        "Nx", "Ny", "Nz", "Nkl", "Nj", "group count", "family count", "input count", "target count"))
    for v, name in ((nx, "Nx"), (ny, "Ny"), (nz, "Nz"), (nkl, "Nkl"), (nj, "Nj"), (ngroups, "group count")):
        _require(v > 0, f"invalid fixture dimension {name}")
    _require(nfam == 2, "spectral-flux fixture must contain wave-f and wave-g")
    _require(nin == 15, "spectral-flux fixture must contain 15 input fields")
    _require(nout == 4, "spectral-flux fixture must contain four targets")
    lx, ly, lz, latitude, scale = (r.scalar("d", name) for name in ("Lx", "Ly", "Lz", "latitude", "pointwise scale"))
    _require(nx == ny and nx % 2 == 0, "the authoritative path requires an even square horizontal grid")
    _require(lx == ly, "the authoritative path requires a square horizontal domain")
    _require(np.isfinite([lx, lz, latitude, scale]).all() and lx > 0 and lz > 0 and scale > 0,
             "spectral-flux fixture contains invalid physical metadata")
    _require(scale == 1.0 / float((nx * ny) ** 2), "spectral-flux fixture pointwise normalization is inconsistent")
    _require(nj == 2 * (nz - 1) // 3, "spectral-flux fixture Nj violates floor(2*(Nz-1)/3)")
    meta = {name: r.string(name) for name in STRINGS}
    _require(meta["fixture_id"] != "", "spectral-flux fixture id is empty")
    _require(meta["repository"] == REPOSITORY, "spectral-flux fixture identifies the wrong WVM repository")
    _require(len(meta["commit"]) == 40, "spectral-flux fixture WVM commit is not a full object id")
    _require(meta["fixture_hash"].startswith("sha256:") and len(meta["fixture_hash"]) == 71,
             "spectral-flux fixture identity is not SHA-256")
    keys = r.array(np.int32, 2 * nkl, "mode keys").reshape(nkl, 2).astype(np.int64)
    vertical = r.array(np.int32, nj, "vertical mode keys")
    group_of = r.array(np.uint32, nkl, "mode group indices").astype(np.int64)
    group_keys = r.array(np.uint64, ngroups, "group keys")
    in_fam = tuple(int(v) for v in r.array(np.uint32, nin, "input field families"))
    out_fam = tuple(int(v) for v in r.array(np.uint32, nout, "target field families"))
    inverse_raw = r.array(np.float64, ngroups * 2 * nz * nj, "inverse operator matrices").reshape(ngroups, 2, nj, nz)
    forward_raw = r.array(np.float64, ngroups * 2 * nz * nj, "forward operator matrices").reshape(ngroups, 2, nz, nj)
    inputs = r.array(np.complex128, nkl * nin * nj, "modal inputs").reshape(nkl, nin, nj)
    targets = r.array(np.complex128, nkl * nout * nj, "modal targets").reshape(nkl, nout, nj)
    _require(r.at == len(r.data), "prepared spectral-flux fixture contains trailing bytes")

    _require(np.array_equal(vertical, np.arange(nj)), "spectral-flux fixture vertical mode keys are not j=0..Nj-1")
    source = {}
    for i, (k, l) in enumerate(keys):
        _require((int(k), int(l)) not in source, "spectral-flux fixture horizontal mode keys are not unique")
        source[(int(k), int(l))] = i
    canonical = retained_keys if retained_keys is not None else _retained_keys(nx, ny)
    _require(len(canonical) == nkl, "spectral-flux fixture retained horizontal mode count is inconsistent")
    order = []
    for key in canonical:
        _require(key in source, "spectral-flux fixture is missing a retained horizontal mode key")
        order.append(source[key])
    _require(len(source) == len(canonical), "spectral-flux fixture contains an unexpected horizontal mode key")
    _require(bool(np.all(group_of < ngroups)), "spectral-flux fixture mode group index is out of range")
    _require(bool(np.all(np.diff(group_of) >= 0)), "spectral-flux fixture mode groups are not contiguous")
    _require(np.array_equal(group_keys[group_of].astype(np.int64), keys[:, 0] ** 2 + keys[:, 1] ** 2),
             "spectral-flux fixture group diagnostic key is inconsistent")
    _require(len(np.unique(group_of)) == ngroups, "spectral-flux fixture does not use every declared mode group")
    _require(bool(np.all(np.diff(group_keys.astype(np.int64)) >= 0)),
             "spectral-flux fixture group diagnostic keys are not nondecreasing")
    _require(in_fam == INPUT_FAMILIES, "spectral-flux fixture input field-to-operator map is inconsistent")
    _require(out_fam == TARGET_FAMILIES, "spectral-flux fixture target-to-operator map is inconsistent")
    for arr, label in ((inverse_raw, "inverse operator"), (forward_raw, "forward operator"), (inputs, "modal input"),
                       (targets, "modal target")):
        _require(bool(np.all(np.isfinite(arr))), f"{label} payload contains a non-finite value")

    order = np.asarray(order)
    inputs = inputs[order]
    targets = targets[order]
    _require(not np.any(inputs[0].imag), "spectral-flux fixture DC modal inputs must be real")
    # Operator groups: runs of retained-order modes that share a file group.
    src_groups = group_of[order]
    starts = np.flatnonzero(np.r_[True, src_groups[1:] != src_groups[:-1]])
    counts = np.diff(np.r_[starts, nkl])
    run_group = src_groups[starts]
    forward = [np.ascontiguousarray(np.transpose(forward_raw[run_group, f], (0, 2, 1))) for f in range(2)]
    inverse = [np.ascontiguousarray(np.transpose(inverse_raw[run_group, f], (0, 2, 1))) for f in range(2)]
    return PreparedFixture(nx, ny, nz, nj, lx, ly, lz, latitude, scale, meta, counts.astype(np.uint64),
                           group_keys[run_group], forward, inverse, in_fam, out_fam, inputs, targets)


def write(path, nx, nz, keys, group_of, group_keys, forward, inverse, inputs, targets, meta=None, lx=1.0, lz=1.0,
          latitude=0.0, input_family=INPUT_FAMILIES, target_family=TARGET_FAMILIES):
    """Write a prepared fixture from data in the file's mode order: keys
    [Nkl][2], group_of [Nkl], group_keys [groups], forward / inverse [family]
    [group][j][z] / [group][z][j], inputs [Nkl][15][Nj], targets [Nkl][4][Nj]."""
    nj = 2 * (nz - 1) // 3
    keys = np.asarray(keys, np.int32).reshape(-1, 2)
    nkl, ngroups = len(keys), len(group_keys)
    m = dict(fixture_id="synthetic", repository=REPOSITORY, commit="0" * 40, generator="synthetic",
             fixture_hash="sha256:" + "0" * 64, normalization="unnormalised FFTW r2c/c2r",
             mode_mapping="retained radial 2/3", derivative_convention="slot map 0..2 U,V,W; 3+3t..5+3t q_t")
    m.update(meta or {})
    out = bytearray(MAGIC)
    out += struct.pack("<IIII", VERSION, BYTE_ORDER, 1, 0)
    out += struct.pack("<9Q", nx, nx, nz, nkl, nj, ngroups, 2, 15, 4)
    out += struct.pack("<5d", lx, lx, lz, latitude, 1.0 / float((nx * nx) ** 2))
    for name in STRINGS:
        raw = m[name].encode("utf-8")
        out += struct.pack("<Q", len(raw)) + raw
    out += keys.astype("<i4").tobytes()
    out += np.arange(nj, dtype="<i4").tobytes()
    out += np.asarray(group_of, "<u4").tobytes()
    out += np.asarray(group_keys, "<u8").tobytes()
    out += np.asarray(input_family, "<u4").tobytes()
    out += np.asarray(target_family, "<u4").tobytes()
    for g in range(ngroups):
        for f in range(2):
            out += np.ascontiguousarray(np.asarray(inverse[f][g]).T, "<f8").tobytes()  # (z, j) at z + Nz j
    for g in range(ngroups):
        for f in range(2):
            out += np.ascontiguousarray(np.asarray(forward[f][g]).T, "<f8").tobytes()  # (j, z) at j + Nj z
    out += np.ascontiguousarray(inputs, "<c16").tobytes()
    out += np.ascontiguousarray(targets, "<c16").tobytes()
    with open(path, "wb") as fh:
        fh.write(bytes(out))
