"""The reference-side C++ adapter (tests/adapter_check.cpp) compiles against
the reference's own headers, and its static_asserts hold: every adapter method
has the parameter, return and const qualification of the reference method it
replaces.  Runs where the reference tree is present (REF in the environment,
else the checkout the golden fixtures were made from); skipped elsewhere."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("REF", "/root/reference")


@pytest.mark.skipif(not os.path.isfile(os.path.join(REF, "include", "skbench", "skbench.hpp")),
                    reason="the reference tree is not present")
@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ is not installed")
def test_adapter_compiles_against_the_reference_headers():
    cmd = ["g++", "-std=c++20", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(REF, "include"), "-I" + os.path.join(REF, "src"),
           os.path.join(ROOT, "tests", "adapter_check.cpp")]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
