"""bench.py --families on CPU: the seeded stand-in wave-f / wave-g operator
families cover the grid's K^2 groups (modes per group summing to the retained
modes, in retained order) with the shapes the two-family flux takes, and are
reproducible; the timed run itself needs a GPU."""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import skb_cuda as S  # noqa: E402
import skb_cuda.fixture as fx  # noqa: E402


def test_synthetic_families_cover_the_k2_groups():
    n, nz = 32, 17
    fam = bench.synthetic_families(n, nz)
    w = S.Workload(n, n, nz, 1)
    groups = S.squared_wavenumber_groups(w)
    assert [int(c) for c in fam["group_modes"]] == [g.mode_count for g in groups]
    assert int(fam["group_modes"].sum()) == len(S.retained_modes(w))
    nj = w.nj
    for f in range(2):
        assert fam["forward"][f].shape == (len(groups), nj, nz)
        assert fam["inverse"][f].shape == (len(groups), nz, nj)
        assert np.all(np.isfinite(fam["forward"][f])) and np.all(np.isfinite(fam["inverse"][f]))
    assert tuple(fam["input_family"]) == fx.INPUT_FAMILIES and tuple(fam["target_family"]) == fx.TARGET_FAMILIES
    again = bench.synthetic_families(n, nz)
    assert all(np.array_equal(a, b) for a, b in zip(fam["forward"] + fam["inverse"], again["forward"] + again["inverse"]))
