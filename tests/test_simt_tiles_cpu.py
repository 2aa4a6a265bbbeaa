"""Host logic of the SIMT grouped vertical GEMM's tile tables (csrc/simt_tiles.hpp):
a C++ checker compiled here with the host compiler covers every (member, column)
exactly once for every member count in both numberings, the member-tile prefix
property that serves partial batches, the member-major launch order and the
90 %-fill rule that picks the numbering."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "spectral-kernel-benchmarks_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_simt_tile_tables(tmp_path):
    exe = tmp_path / "simt_tiles_check"
    src = os.path.join(ROOT, "tests", "simt_tiles_check.cpp")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, src, "-o", str(exe)], check=True, timeout=120)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"
