"""Synthetic prepared spectral-flux fixtures for the tests (the authoritative
WVM exports are not available here).  The data are seeded: K^2 groups split
into two "floating" groups sharing a key where they hold at least three modes,
modes stored in the file in reverse order within each group, wave-f / wave-g
matrices drawn per group, modal inputs uniform in [-0.125, 0.125] with a real
DC mode, and expected targets computed by the oracle's two-family flux."""

import numpy as np

import skb_cuda.fixture as fx
from oracle import oracle as orc


def families_canonical(n, nz, seed):
    """Floating groups over the retained modes (retainedHorizontalModes order)
    and seeded matrices per group and family."""
    modes = orc.retained_modes(n, n)
    keys, first, counts = orc.k2_groups(n, n)
    group_modes, group_keys = [], []
    for key, c in zip(keys, counts):
        parts = [c] if c < 3 else [c // 2, c - c // 2]
        group_modes += parts
        group_keys += [int(key)] * len(parts)
    nj = 2 * (nz - 1) // 3
    rng = np.random.default_rng(seed)
    G = len(group_modes)
    forward = [rng.standard_normal((G, nj, nz)) / np.sqrt(nz) for _ in range(2)]
    inverse = [rng.standard_normal((G, nz, nj)) / np.sqrt(nj) for _ in range(2)]
    fam = {"group_modes": np.asarray(group_modes, np.uint64), "forward": forward, "inverse": inverse,
           "input_family": fx.INPUT_FAMILIES, "target_family": fx.TARGET_FAMILIES}
    return modes, fam, np.asarray(group_keys, np.uint64)


def make(path, n, nz, seed=7, workers=4):
    """Write a fixture to `path`; return (canonical families, inputs, expected)."""
    modes, fam, group_keys = families_canonical(n, nz, seed)
    H = len(modes)
    nj = 2 * (nz - 1) // 3
    rng = np.random.default_rng(seed + 1)
    inputs = rng.uniform(-0.125, 0.125, (H, 15, nj)) + 1j * rng.uniform(-0.125, 0.125, (H, 15, nj))
    inputs[0].imag = 0.0
    expected = orc.flux(n, nz, inputs.reshape(-1), targets=4, modes=modes, workers=workers,
                        families=fam).reshape(H, 4, nj)
    # File order: reverse within each group.
    counts = fam["group_modes"].astype(np.int64)
    first = np.r_[0, np.cumsum(counts)[:-1]]
    order = np.concatenate([np.arange(f0 + c - 1, f0 - 1, -1) for f0, c in zip(first, counts)])
    group_of = np.repeat(np.arange(len(counts)), counts)
    keys = np.stack([modes.k, modes.l], axis=1)
    fx.write(path, n, nz, keys[order], group_of, group_keys, fam["forward"], fam["inverse"], inputs[order],
             expected[order])
    return fam, inputs, expected
