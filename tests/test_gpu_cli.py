"""skbench-cuda run / validate on the GPU: every kernel writes a report whose
JSON keys are the reference writer's (the golden schema sample produced by the
reference's own json.cpp) and whose CSV has the reference's nine columns, and
`validate` passes against the direct transforms."""

import csv
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "spectral-kernel-benchmarks_b200", "skbench-cuda")
GOLDEN = os.path.join(ROOT, "tests", "golden")

pytestmark = pytest.mark.gpu


def keys_match(sample, got, path="$"):
    """Every key of the reference sample exists in `got`, recursively."""
    if isinstance(sample, dict):
        assert isinstance(got, dict), path
        for k, v in sample.items():
            assert k in got, path + "." + k
            keys_match(v, got[k], path + "." + k)
    elif isinstance(sample, list) and sample and got:
        keys_match(sample[0], got[0], path + "[0]")


def run(tmp_path, *args):
    out_json = tmp_path / "report.json"
    proc = subprocess.run([CLI, "run", *args, "--output", str(out_json)], capture_output=True, text=True,
                          timeout=600)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    report = json.loads(out_json.read_text())
    with open(out_json.with_suffix(".csv")) as fh:
        rows = list(csv.reader(fh))
    return report, rows


@pytest.mark.parametrize("args", [
    ("--kernel", "fft"),
    ("--kernel", "2d-rfft", "--precision", "fp32"),
    ("--kernel", "pruned-horizontal"),
    ("--kernel", "pruned-horizontal", "--precision", "fp32"),
    ("--kernel", "vertical-gemm", "--vertical-gemm-family", "common"),
    ("--kernel", "vertical-gemm", "--vertical-gemm-family", "k2-grouped", "--vertical-gemm-precision", "fp32"),
    ("--kernel", "pointwise-advection"),
    ("--kernel", "production-lifetime-flux", "--flux-mode", "fp64-plain", "--nx", "32", "--ny", "32", "--nz", "9"),
    ("--kernel", "production-lifetime-flux", "--flux-mode", "split-tf32x3", "--nx", "64", "--ny", "64", "--nz",
     "17", "--members", "2"),
    ("--kernel", "production-lifetime-flux", "--flux-mode", "split-tf32x3", "--nx", "64", "--ny", "64", "--nz",
     "17", "--members", "2", "--autotune", "on"),
    ("--kernel", "spectral-pipeline", "--nx", "32", "--ny", "32", "--nz", "9"),
    ("--kernel", "spectral-pipeline", "--precision", "fp32", "--nx", "32", "--ny", "32", "--nz", "9"),
], ids=lambda a: "-".join(a[1::2]))
def test_run_writes_the_reference_schema(tmp_path, args):
    autotune = "--autotune" in args
    if autotune:
        args = tuple(a for a in args if a != "on")
    report, rows = run(tmp_path, "--profile", "smoke", *args)
    if autotune:
        cfg = report["providers"][0]["planning"]["configuration"]
        assert "autotuned: flux.tc_gemm.unit_tiles inverse" in cfg, cfg
    with open(os.path.join(GOLDEN, "reference_report.json")) as fh:
        keys_match(json.load(fh), report)
    assert report["status"] == "passed"
    provider = report["providers"][0]
    assert provider["id"] == "cuda"
    assert provider["correctness"] and all(m["passed"] for m in provider["correctness"])
    assert any(t["scope"] == "primitive" and t["medianSeconds"] > 0 for t in provider["timings"])
    assert rows[0] == ["run_id", "provider", "scope", "stage", "direction", "state", "bytes_moved", "sample_index",
                       "seconds"]
    assert len(rows) > 1 and all(len(r) == 9 for r in rows)


@pytest.mark.parametrize("args", [
    ("--profile", "smoke"),
    ("--profile", "smoke", "--precision", "fp32"),
    ("--profile", "quick", "--samples", "3", "--warmups", "1"),
    ("--profile", "wvm-historical-512-nz129-f4", "--samples", "3", "--warmups", "1"),
], ids=lambda a: "-".join(a[1::2]))
def test_constant_stratification_vertical_records(tmp_path, args):
    """runConstantStratificationVerticalBenchmark's report shape
    (src/constant_stratification.cpp:481-648): a full-half and a retained
    compact record, seven timings each, two direct-oracle checks on both and
    the two compact-versus-full schedule checks on the compact one."""
    report, rows = run(tmp_path, "--kernel", "constant-stratification-vertical", *args)
    with open(os.path.join(GOLDEN, "reference_report.json")) as fh:
        keys_match(json.load(fh), report)
    assert report["status"] == "passed"
    assert report["workload"]["fields"] == 4
    full, compact = report["providers"]
    assert full["id"] == "cuda-wvm-type1-full-half" and compact["id"] == "cuda-wvm-type1-retained-compact"
    for p, checks in ((full, 2), (compact, 4)):
        assert len(p["correctness"]) == checks and all(m["passed"] for m in p["correctness"])
        stages = {(t["scope"], t["stage"], t["direction"]) for t in p["timings"]}
        assert ("primitive", "raw DCT-I one complex channel", "inverse") in stages
        assert ("primitive", "raw DST-I one complex interior channel", "forward") in stages
        assert ("adapter-component", "WVM forward DST-I normalization and endpoints", "forward") in stages
        total = [t for t in p["timings"] if t["scope"] == "uninstrumented-total"]
        assert len(total) == 1 and total[0]["medianSeconds"] > 0
    assert len(rows) > 1 and all(len(r) == 9 for r in rows)


def test_validate_passes():
    proc = subprocess.run([CLI, "validate"], capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stdout + proc.stderr
    assert "validation passed" in proc.stdout
    assert proc.stdout.count("cuda/") == 10 and proc.stdout.count("cuda-pruned/") == 10
    assert "cuda-flux/split-tf32x3/32x32x9" in proc.stdout


@pytest.mark.parametrize("mode", ["fp64-plain", "split-tf32x3"])
def test_authoritative_fixture_run(tmp_path, mode):
    """--spectral-flux-fixture: the two-family flux against the fixture's
    expected targets (a synthetic fixture in the prepared format)."""
    import sys

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from synthetic_fixture import make

    path = tmp_path / "fixture.bin"
    make(path, 16, 9)
    report, rows = run(tmp_path, "--kernel", "production-lifetime-flux", "--profile", "smoke", "--nx", "16", "--ny",
                       "16", "--nz", "9", "--flux-mode", mode, "--spectral-flux-fixture", str(path))
    assert report["status"] == "passed"
    provider = report["providers"][0]
    assert len(provider["correctness"]) == 1 and provider["correctness"][0]["passed"]
    assert "synthetic" in provider["planning"]["configuration"]


def test_streaming_options_are_recorded(tmp_path):
    """The reference's streaming-provider knobs run the flux unchanged and are
    recorded in the provider's ledger."""
    report, _ = run(tmp_path, "--kernel", "production-lifetime-flux", "--flux-mode", "fp64-plain", "--nx", "32",
                    "--ny", "32", "--nz", "9", "--boundary-policy", "streaming-pruned-compact-split",
                    "--streaming-tile-width", "16")
    assert report["status"] == "passed"
    ledger = report["providers"][0]["componentLedger"]
    entry = next(e for e in ledger if e["stage"] == "streaming preparation options")
    assert "streaming-pruned-compact-split" in entry["detail"] and "tile width 16" in entry["detail"]
