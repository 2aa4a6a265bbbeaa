"""The skbench-cuda command line without a GPU: argument handling, profile
list, exit codes (main.cpp:242-245 maps errors to 2) and `compare` over the
reference writer's own CSV sample."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "spectral-kernel-benchmarks_b200", "skbench-cuda")
GOLDEN = os.path.join(ROOT, "tests", "golden")

pytestmark = pytest.mark.skipif(not os.path.exists(CLI), reason="skbench-cuda is not built")


def cli(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60)


def test_list_names_the_reference_profiles_and_kernels():
    out = cli("list")
    assert out.returncode == 0
    for name in ("smoke: 8x8, Nz=7, fields=2", "quick: 256x256, Nz=65, fields=3",
                 "wvm-historical-512-nz129-f4: 512x512, Nz=129, fields=4", "wvm-large-1024-nz129-f4"):
        assert name in out.stdout
    for kernel in ("fft (alias 2d-rfft)", "pruned-horizontal", "vertical-gemm", "pointwise-advection",
                   "production-lifetime-flux", "spectral-pipeline", "constant-stratification-vertical"):
        assert kernel in out.stdout


@pytest.mark.parametrize("args", [(), ("bogus",), ("list", "extra"), ("run", "--kernel", "bogus"),
                                  ("run", "--profile", "nope"), ("run", "--warmups"), ("validate", "--x"),
                                  ("compare",)])
def test_bad_arguments_exit_2(args):
    out = cli(*args)
    assert out.returncode == 2
    assert args == () or "skbench-cuda:" in out.stderr


def test_compare_reads_the_reference_csv():
    out = cli("compare", "--input", os.path.join(GOLDEN, "reference_report.csv"))
    assert out.returncode == 0
    lines = out.stdout.strip().splitlines()
    assert lines[0] == "provider\tscope\tstage\tdirection\tmedian_ms\tsamples"
    assert lines[1].split("\t") == ["sample", "primitive", "stage", "forward", "1500.000000", "2"]


def test_bad_fixture_exits_2(tmp_path):
    """The prepared fixture is validated before any device work."""
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"SKFXP002" + bytes(64))
    out = cli("run", "--kernel", "production-lifetime-flux", "--spectral-flux-fixture", str(bad))
    assert out.returncode == 2
    assert "wrong magic" in out.stderr
    out = cli("run", "--kernel", "fft", "--spectral-flux-fixture", str(bad))
    assert out.returncode == 2 and "valid only for production-lifetime-flux" in out.stderr


@pytest.mark.parametrize("args,message", [
    (("--kernel", "fft", "--streaming-inverse-policy", "active-reset"), "production-lifetime-flux only"),
    (("--kernel", "production-lifetime-flux", "--streaming-inverse-policy", "compact-preserved"),
     "needs a prepared fixture"),
    (("--kernel", "production-lifetime-flux", "--streaming-inverse-policy", "sideways"), "expected full-zero"),
    (("--kernel", "production-lifetime-flux", "--boundary-policy", "wvm-packed-split"),
     "wvm-direct, streaming-pruned-compact-split"),
    (("--kernel", "spectral-pipeline", "--boundary-policy", "pruned-compact-interleaved"), "plane-major-fused-split"),
])
def test_streaming_options_are_checked_like_the_reference(args, message):
    """--boundary-policy / --streaming-tile-width / --streaming-inverse-policy
    (the reference's streaming-provider knobs) are accepted, and the values the
    reference refuses for a kernel are refused with exit 2 before device work."""
    out = cli("run", *args)
    assert out.returncode == 2, out.stdout + out.stderr
    assert message in out.stderr


def test_tile_width_other_than_sixteen_is_refused_for_a_prepared_fixture(tmp_path):
    path = tmp_path / "f.bin"
    path.write_bytes(b"SKFXP001")
    out = cli("run", "--kernel", "production-lifetime-flux", "--spectral-flux-fixture", str(path),
              "--streaming-tile-width", "8")
    assert out.returncode == 2 and "16-plane tiles" in out.stderr
