#!/usr/bin/env python
"""Benchmark of the composed antialiased flux on B200.

Workload: the full 15 -> 4 flux (inverse K^2-grouped vertical GEMM, inverse
pruned 2-D transforms, pointwise advection, forward pruned transforms with 2/3
truncation, forward vertical GEMM) at 512 x 512 horizontal, Nz = 129, 4 target
fields, 8 ensemble members per launch, replayed from one CUDA graph.  Metric:
flux evaluations per second (one evaluation = one member's 15 -> 4 flux).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--mode split|fp32|fp64]
    python bench.py --impl reference ...     # CPU arm, rank 0 only
    python bench.py --serve [--serve-rate R]  # serving benchmark on its own line
    python bench.py --profile-run --members 2 --repeat 1   # device path for a kernel profiler

The default line also times the FP64-plain flux on the same inputs (the
ratio's denominator) and runs a short serving pass: the same seeded Poisson
stream of mixed requests through the split and the FP64-plain paths, whose
p50 / p99 latencies it reports.

Under torchrun every rank runs an independent replica (the path shards over
members with no exchange); a gloo barrier brackets the timed region and the
step time is the max over ranks.  Prints one JSON line on rank 0.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "spectral-kernel-benchmarks_b200"))

import numpy as np  # noqa: E402

METRIC = "flux evals/s (512²×129,f4) split-prec vs FP64-plain at ≤1e-6 rel err; p99 ms"
UNIT = "evals/s"
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 1024 * 1024


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    p.add_argument("--mode", choices=["split", "bf16x3", "fp32", "fp64"], default="split",
                   help="split: split-TF32x3 tensor-core GEMMs; bf16x3: split-BF16x3 ones")
    p.add_argument("--n", type=int, default=512)
    p.add_argument("--nz", type=int, default=129)
    p.add_argument("--members", type=int, default=8)
    p.add_argument("--e2e-steps", type=int, default=10)
    p.add_argument("--skip-cpu-baseline", action="store_true")
    p.add_argument("--skip-e2e", action="store_true")
    p.add_argument("--skip-fp64", action="store_true",
                   help="do not time the FP64-plain flux beside the split one")
    p.add_argument("--skip-serve-pass", action="store_true",
                   help="do not run the short same-stream serving pass (split and FP64-plain)")
    p.add_argument("--profile-run", action="store_true",
                   help="for a kernel profiler: run the device path (no graph) --repeat times, print the "
                        "per-stage event timing of one more run as JSON, and exit")
    p.add_argument("--repeat", type=int, default=1)
    p.add_argument("--no-stage-times", action="store_true", help="with --profile-run: skip the extra timed run")
    p.add_argument("--autotune", action="store_true", help="with --profile-run: apply the autotuner's shapes first")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch shapes instead of the autotuner's choices")
    p.add_argument("--families", action="store_true",
                   help="the authoritative two-family flux (wave-f / wave-g operators) with seeded stand-in "
                        "matrices over the K^2 groups")
    p.add_argument("--serve", action="store_true",
                   help="serving benchmark: Poisson arrivals over mixed grid sizes with resident states")
    p.add_argument("--serve-requests", type=int, default=600)
    p.add_argument("--serve-rate", type=float, default=400.0, help="mean arrivals per second")
    p.add_argument("--serve-batch", type=int, default=8)
    p.add_argument("--serve-states", type=int, default=8, help="resident member states per size class")
    p.add_argument("--serve-pass-rate", type=float, default=150.0,
                   help="arrival rate of the serving pass that runs with the default benchmark")
    p.add_argument("--serve-pass-requests", type=int, default=300)
    return p.parse_args()


# ------------------------------------------------------------ distribution

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, value):
        if not self.pg:
            return value
        import torch

        t = torch.tensor([float(value)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a while to print its first sample: wait for it
            # (at most 3 s), then keep only the samples of the timed region.
            t0 = time.time()
            while not self.lines and self.proc.poll() is None and time.time() - t0 < 3.0:
                time.sleep(0.005)
            self.lines.clear()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self):
        sm, smax, reasons = [], None, set()
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                  parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ inputs

def mode_wavenumbers(n):
    """(k, l) of the retained radial-2/3 modes, from the library's own mode table."""
    import skb_cuda as S

    modes = S.retained_modes(S.Workload(n, n, 1, 1))
    return (np.array([m.k for m in modes], dtype=np.float64), np.array([m.l for m in modes], dtype=np.float64))


def power_law_inputs(n, nz, members, targets=4, seed=129):
    """Seeded k^-3 power-law modal spectra: amplitude (1 + |k|^2)^(-3/2) times a
    uniform random phase, for every (member, mode, field, j)."""
    k, l = mode_wavenumbers(n)
    nj = 2 * (nz - 1) // 3
    fields = 3 + 3 * targets
    rng = np.random.default_rng(seed)
    amp = (1.0 + k * k + l * l) ** -1.5
    shape = (members, len(k), fields, nj)
    phase = rng.uniform(0.0, 2.0 * np.pi, shape)
    mag = rng.uniform(0.5, 1.5, shape)
    x = (amp[None, :, None, None] * mag) * np.exp(1j * phase)
    dc = (k == 0) & (l == 0)
    x[:, dc, :, :] = x[:, dc, :, :].real
    return np.ascontiguousarray(x.reshape(-1))


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel_stage):
    """Per-launch DRAM bytes of a stage from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "flux_traffic.json")
    try:
        with open(path) as fh:
            table = json.load(fh)
        return table.get(kernel_stage)
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------- CUDA arm

def synthetic_families(n, nz, seed=5):
    """Seeded stand-ins for the WVM wave-f / wave-g operator families (the
    prepared WVM exports are not available): over the grid's K^2 groups, per
    family and group, Gaussian forward [j][z] and inverse [z][j] matrices
    scaled by 1/sqrt(inner size), with the reference's field-to-family maps."""
    import skb_cuda as S
    import skb_cuda.fixture as fx

    w = S.Workload(n, n, nz, 1)
    counts = np.array([g.mode_count for g in S.squared_wavenumber_groups(w)], dtype=np.uint64)
    rng = np.random.default_rng(seed)
    groups, nj = len(counts), w.nj
    return {"group_modes": counts,
            "forward": [rng.standard_normal((groups, nj, nz)) / np.sqrt(nz) for _ in range(2)],
            "inverse": [rng.standard_normal((groups, nz, nj)) / np.sqrt(nj) for _ in range(2)],
            "input_family": fx.INPUT_FAMILIES, "target_family": fx.TARGET_FAMILIES}


def timed_replays(S, flux, steps, dist):
    """Device time of `steps` graph replays on the flux's stream (CUDA events),
    bracketed by a barrier and a device synchronisation; max over ranks."""
    stream = flux.stream
    timer = S.Timer()
    dist.barrier()
    S.synchronize()
    timer.start(stream)
    for _ in range(steps):
        flux.replay_graph()
    timer.stop(stream)
    S.synchronize()
    dist.barrier()
    return dist.max(timer.elapsed_ms() / steps)


def fp64_plain_leg(S, args, x, families, dist):
    """The FP64-plain flux (the north-star denominator) on the same inputs, by
    the same method as the split line: graph capture, warm-up, `steps` timed
    replays.  Returns (evals/s, ms per step, its output)."""
    ref_flux = S.Flux(args.n, args.nz, targets=4, members=args.members, mode=S.FLUX_FP64_PLAIN, families=families)
    din = S.DeviceArray.from_numpy(np.ascontiguousarray(x, dtype=np.complex128))
    dout = S.DeviceArray(ref_flux.output_elements * 16)
    ref_flux.execute_device(din.ptr, dout.ptr)
    ref_flux.capture_graph(din.ptr, dout.ptr)
    for _ in range(args.warmup):
        ref_flux.replay_graph()
    S.synchronize()
    ms = timed_replays(S, ref_flux, args.steps, dist)
    ref_flux.check_device()
    out = dout.download(np.complex128, ref_flux.output_elements)
    ref_flux.close()
    din.free()
    dout.free()
    return dist.world * args.members * 1000.0 / ms, ms, out


def profile_run(args, dist):
    """Device-path executions for a kernel profiler (no graph, so each launch
    is visible), then the per-stage event timing of one more execution."""
    import skb_cuda as S

    S.set_device(dist.local)
    mode = {"split": S.FLUX_SPLIT_TF32X3, "bf16x3": S.FLUX_SPLIT_BF16X3, "fp32": S.FLUX_FP32,
            "fp64": S.FLUX_FP64_PLAIN}[args.mode]
    families = synthetic_families(args.n, args.nz) if args.families else None
    flux = S.Flux(args.n, args.nz, targets=4, members=args.members, mode=mode, families=families)
    x = power_law_inputs(args.n, args.nz, args.members, seed=129 + dist.rank)
    din = S.DeviceArray.from_numpy(x.astype(flux.device_dtype))
    dout = S.DeviceArray(flux.output_elements * np.dtype(flux.device_dtype).itemsize)
    tuned = flux.autotune(din.ptr, dout.ptr) if args.autotune else {}
    for _ in range(args.repeat):
        flux.execute_device(din.ptr, dout.ptr)
    S.synchronize()
    flux.check_device()
    if args.no_stage_times or dist.rank != 0:
        return None
    return {"profile_run": {"n": args.n, "nz": args.nz, "members": args.members, "mode": args.mode,
                            "repeat": args.repeat, "autotune": {k: v[0] for k, v in tuned.items()}},
            "stages": flux.profile(din.ptr, dout.ptr)}


def cuda_arm(args, dist):
    import skb_cuda as S

    S.set_device(dist.local)
    mode = {"split": S.FLUX_SPLIT_TF32X3, "bf16x3": S.FLUX_SPLIT_BF16X3, "fp32": S.FLUX_FP32,
            "fp64": S.FLUX_FP64_PLAIN}[args.mode]
    families = synthetic_families(args.n, args.nz) if args.families else None
    flux = S.Flux(args.n, args.nz, targets=4, members=args.members, mode=mode, families=families)
    mode_name = {"split": "split-tf32x3", "bf16x3": "split-bf16x3"}.get(args.mode, args.mode)
    dtype = flux.device_dtype
    x = power_law_inputs(args.n, args.nz, args.members, seed=129 + dist.rank)
    din = S.DeviceArray.from_numpy(x.astype(dtype))
    dout = S.DeviceArray(flux.output_elements * np.dtype(dtype).itemsize)

    # Launch shapes from the project autotuner (measured on these buffers,
    # outside the timed region), then warm-up through the graph path
    # (captures once, then replays).
    tuned, tune_s = {}, 0.0
    if not args.no_autotune:
        t0 = time.perf_counter()
        tuned = flux.autotune(din.ptr, dout.ptr)
        tune_s = time.perf_counter() - t0
    flux.execute_device(din.ptr, dout.ptr)
    flux.capture_graph(din.ptr, dout.ptr)
    for _ in range(args.warmup):
        flux.replay_graph()
    S.synchronize()

    with ClockSampler(dist.local) as clocks:
        ms_max = timed_replays(S, flux, args.steps, dist)
    flux.check_device()
    value = dist.world * args.members * 1000.0 / ms_max

    stages = flux.profile(din.ptr, dout.ptr)
    info = flux.info()

    # The FP64-plain flux on the same inputs, timed the same way (the ratio's
    # denominator), and this run's error against it.
    rel_err, fp64 = None, None
    if mode != S.FLUX_FP64_PLAIN:
        flux.replay_graph()
        S.synchronize()
        out = dout.download(dtype, flux.output_elements).astype(np.complex128)
        if args.skip_fp64:
            ref_flux = S.Flux(args.n, args.nz, targets=4, members=args.members, mode=S.FLUX_FP64_PLAIN,
                              families=families)
            ref = ref_flux.execute(x)
            ref_flux.close()
        else:
            with ClockSampler(dist.local) as fp64_clocks:
                fp64_value, fp64_ms, ref = fp64_plain_leg(S, args, x, families, dist)
            fp64 = {"evals_per_s": fp64_value, "ms_per_step": fp64_ms, "steps": args.steps,
                    "warmup": args.warmup, "dtype": "f64", "clocks": fp64_clocks.summary()}
        num = float(np.linalg.norm(out - ref))
        den = float(np.linalg.norm(ref))
        rel_err = num / den if den else num
        if fp64 is not None:
            fp64["split_rel_l2_err"] = rel_err
            fp64["split_max_rel_err"] = float(np.max(np.abs(out - ref)) / max(1.0, float(np.max(np.abs(ref)))))

    # End to end through the public host API: pinned FP64 host arrays, H2D,
    # compute, D2H every step.
    e2e = None
    if not args.skip_e2e:
        hin = S.PinnedArray(np.complex128, flux.input_elements)
        hout = S.PinnedArray(np.complex128, flux.output_elements)
        hin.array[:] = x
        flux.execute_host_ptr(hin.ptr, hout.ptr)
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            flux.execute_host_ptr(hin.ptr, hout.ptr)
        t1 = time.perf_counter()
        dist.barrier()
        e2e_ms = dist.max((t1 - t0) * 1000.0 / args.e2e_steps)
        e2e = {"value": dist.world * args.members * 1000.0 / e2e_ms, "unit": UNIT,
               "h2d_bytes_per_step": int(hin.array.nbytes), "d2h_bytes_per_step": int(hout.array.nbytes),
               "ms_per_step": e2e_ms, "steps": args.e2e_steps}
        hin.free()
        hout.free()

    # Serving: the same seeded Poisson stream of mixed requests through the
    # split and the FP64-plain paths (p50 / p99 latency of the metric).
    serving = None
    if not args.skip_serve_pass and not args.families:
        flux.close()
        din.free()
        dout.free()
        serving = {"arrival_rate_per_s": args.serve_pass_rate, "requests": args.serve_pass_requests,
                   "mix": "40% 128x128xNz33 12->3, 40% 256x256xNz65 12->3, 20% 512x512xNz129 15->4",
                   "max_batch": args.serve_batch, "resident_states_per_class": 2}
        for name, m in (("split", S.FLUX_SPLIT_TF32X3), ("fp64", S.FLUX_FP64_PLAIN)):
            r = serving_run(S, m, args.serve_pass_rate, args.serve_pass_requests, args.serve_batch, 2, dist)
            serving[name] = {k: r[k] for k in ("p50_ms", "p99_ms", "throughput_evals_per_s", "classes", "batches")}

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.skip_cpu_baseline:
        cpu = cpu_baseline(args)

    if dist.rank != 0:
        return None
    peak, peak_kind = measured_peak()
    dominant = max(stages, key=lambda s: s["ms"])
    per_launch_ms = dominant["ms"] / max(1, dominant["launches"])
    per_launch_bytes = dominant["bytes"] / max(1, dominant["launches"])
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9
    # The compute side of the same kernel: measured SIMT FMA peaks, and for the
    # fused row kernel its nominal flops per launch, 19 real transforms of
    # 2.5 N log2 N and 4 targets x 6 flops per point, per (row, plane, member).
    simt = None
    try:
        f32, f64 = S.simt_peaks()
        simt = {"fp32_tflops": f32, "fp64_tflops": f64,
                "how": "independent FMA chains at full occupancy, best of 3 (skb_measure_simt_peaks)"}
    except (RuntimeError, ValueError, MemoryError):
        pass
    compute = None
    if simt and dominant["name"] == "rows_flux_fused":
        per_row = (19 * 2.5 * args.n * np.log2(args.n) + 4 * 6 * args.n)
        flops = per_row * args.n * args.nz * args.members
        tf = flops / (per_launch_ms * 1e-3) / 1e12
        peak_c = simt["fp64_tflops"] if mode == S.FLUX_FP64_PLAIN else simt["fp32_tflops"]
        compute = {"flops_per_launch": flops, "achieved_tflops": tf, "peak_tflops": peak_c,
                   "frac": tf / peak_c if peak_c else None, "peak_kind": "measured (SIMT FMA)"}
    total_ms = sum(s["ms"] for s in stages)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {S.FLUX_FP64_PLAIN: "f64", S.FLUX_FP32: "f32", S.FLUX_SPLIT_BF16X3: "bf16x3+f32"}.get(mode, "tf32x3+f32"),
        "data": "synthetic (seeded k^-3 power-law modal spectra, "
                + ("seeded Gaussian wave-f / wave-g operator families over the K^2 groups)" if families else
                   "K^2 pair-rotation vertical family)"),
        "config": {"workload": f"15->4 {'two-family ' if families else ''}flux {args.n}x{args.n}, Nz={args.nz}, "
                               f"4 targets, {args.members} members per launch, CUDA graph replay",
                   "n": args.n, "nz": args.nz, "targets": 4, "members_per_gpu": args.members, "mode": mode_name,
                   "evals_per_step_per_gpu": args.members, "l2": "inputs larger than L2 (%.2f GB modal input)"
                   % (din.nbytes / 1e9), "parallelism": f"replicas x{dist.world}",
                   "autotune": {"seconds": round(tune_s, 3),
                                "choices": {k.split(" | ")[0]: v[0] for k, v in tuned.items()}}},
        "rel_err_vs_fp64": rel_err,
        "fp64_plain": fp64,
        "split_over_fp64": (value / fp64["evals_per_s"]) if fp64 else None,
        "p99_ms": serving["split"]["p99_ms"] if serving else None,
        "serving": serving,
        "roofline": {"bound": "hbm", "kernel": dominant["name"], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": ncu_traffic(dominant["name"]),
                     "algorithmic_bytes_per_launch": per_launch_bytes, "launch_ms": per_launch_ms,
                     "compute": compute},
        "simt_peaks": simt,
        "stages": [{"name": s["name"], "ms": round(s["ms"], 4), "share": round(s["ms"] / total_ms, 4),
                    "launches": s["launches"], "GBps": (s["bytes"] / (s["ms"] * 1e-3) / 1e9) if s["ms"] else None}
                   for s in stages],
        "e2e": e2e,
        "gpu_launches": int(info["launches_per_execution"]) * args.steps,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    return line


# ---------------------------------------------------------------- serving

# Size classes of the serving mix: (n, Nz, targets, share of arrivals);
# targets 3 is the 12 -> 3 variant, 4 the full 15 -> 4 flux.
SERVE_CLASSES = [(128, 33, 3, 0.4), (256, 65, 3, 0.4), (512, 129, 4, 0.2)]


def serving_run(S, mode, rate, requests, batch, states_per_class, dist, classes_mix=None):
    """Requests with seeded exponential inter-arrival times (`rate` per second)
    pick a size class by the mix and a resident member state of that class; the
    server batches what queues per class.  Latency = submit -> result in host
    memory.  The stream (classes, gaps, states) depends only on the seeds, so
    two modes see the same requests at the same times."""
    mix = classes_mix or SERVE_CLASSES
    classes = [(n, nz, t, batch, mode) for n, nz, t, _ in mix]
    # The slots' pipelines take their launch shapes from the project tuning
    # cache: tune each class once, at the slots' batch size, before serving.
    for n, nz, t, _ in mix:
        f = S.Flux(n, nz, targets=t, members=batch, mode=mode)
        dtype = f.device_dtype
        din = S.DeviceArray.from_numpy(power_law_inputs(n, nz, batch, targets=t, seed=31).astype(dtype))
        dout = S.DeviceArray(f.output_elements * np.dtype(dtype).itemsize)
        f.autotune(din.ptr, dout.ptr)
        f.close()
        din.free()
        dout.free()
    server = S.Server(classes, hbm_budget_bytes=64 << 30, max_slots_per_class=2)
    states = []
    for c, (n, nz, t, _) in enumerate(mix):
        states.append([server.load_state(c, power_law_inputs(n, nz, 1, targets=t, seed=1000 * c + i + 977 * dist.rank))
                       for i in range(states_per_class)])
    rng = np.random.default_rng(7 + dist.rank)
    picks = rng.choice(len(mix), size=requests, p=[c[3] for c in mix])
    gaps = rng.exponential(1.0 / rate, size=requests)
    outputs = [S.PinnedArray(np.complex128, server.sizes[c][1]) for c in range(len(mix)) for _ in range(2)]
    # Warm-up: every class once, alone.
    for c in range(len(mix)):
        server.wait(server.submit_state(states[c][0], outputs[2 * c].array), timeout=300)
    base = server.stats()
    dist.barrier()
    tickets = []
    t0 = time.perf_counter()
    due = t0
    with ClockSampler(dist.local) as clocks:
        for i, c in enumerate(picks):
            due += gaps[i]
            while True:
                now = time.perf_counter()
                if now >= due:
                    break
                if due - now > 2e-4:
                    time.sleep(due - now - 1e-4)
            # Two pinned result buffers per class, reused: the results of
            # this benchmark are not read, only their arrival times.
            tickets.append((c, server.submit_state(states[c][i % states_per_class], outputs[2 * c + i % 2].array)))
        lat = [(c, server.wait(t, timeout=600)[1]) for c, t in tickets]
        t1 = time.perf_counter()
    stats = server.stats()
    server.close()
    for o in outputs:
        o.free()
    all_ms = np.array([x for _, x in lat])
    span = t1 - t0
    per_class = {}
    for c, (n, nz, t, share) in enumerate(mix):
        v = np.array([x for k, x in lat if k == c])
        per_class[f"{n}x{n}xNz{nz}_f{t}"] = {
            "requests": int(v.size), "p50_ms": float(np.percentile(v, 50)) if v.size else None,
            "p99_ms": float(np.percentile(v, 99)) if v.size else None,
            "evals_per_s": float(v.size / span)}
    return {"p50_ms": float(np.percentile(all_ms, 50)), "p99_ms": float(np.percentile(all_ms, 99)),
            "mean_ms": float(np.mean(all_ms)), "throughput_evals_per_s": float(len(all_ms) / span),
            "classes": per_class, "batches": stats["batches"] - base["batches"],
            "server": {"batches": stats["batches"] - base["batches"], "slots": stats["slots"],
                       "slot_bytes": stats["slot_bytes"], "state_bytes": stats["state_bytes"]},
            "clocks": clocks.summary()}


def serve_arm(args, dist):
    """The serving benchmark on its own line (p99 latency as the value)."""
    import skb_cuda as S

    S.set_device(dist.local)
    mode = {"split": S.FLUX_SPLIT_TF32X3, "bf16x3": S.FLUX_SPLIT_BF16X3, "fp32": S.FLUX_FP32,
            "fp64": S.FLUX_FP64_PLAIN}[args.mode]
    r = serving_run(S, mode, args.serve_rate, args.serve_requests, args.serve_batch, args.serve_states, dist)
    if dist.rank != 0:
        return None
    mode_name = {"split": "split-tf32x3", "bf16x3": "split-bf16x3"}.get(args.mode, args.mode)
    return {
        "metric": "serving p99 latency, mixed flux requests (40% 128²×33 f3, 40% 256²×65 f3, 20% 512²×129 f4)",
        "value": r["p99_ms"], "unit": "ms", "n_gpus": dist.world,
        "steps": args.serve_requests, "warmup": len(SERVE_CLASSES), "ms_per_step": r["mean_ms"],
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": {S.FLUX_FP64_PLAIN: "f64", S.FLUX_FP32: "f32", S.FLUX_SPLIT_BF16X3: "bf16x3+f32"}.get(mode, "tf32x3+f32"),
        "data": "synthetic (seeded k^-3 power-law resident states, seeded Poisson arrivals)",
        "config": {"workload": "continuous-batching flux server", "mode": mode_name,
                   "arrival_rate_per_s": args.serve_rate, "requests": args.serve_requests,
                   "max_batch": args.serve_batch, "resident_states_per_class": args.serve_states,
                   "parallelism": f"replicas x{dist.world}"},
        "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
        "throughput_evals_per_s": r["throughput_evals_per_s"], "classes": r["classes"],
        "server": r["server"], "clocks": r["clocks"],
    }


# ------------------------------------------------------------- CPU arms

def cpu_flux_once(n, nz, seed, workers):
    """One member's 15 -> 4 flux on the host: threaded pocketfft FP64 transforms,
    per-group BLAS GEMMs and the threaded pointwise product (oracle port)."""
    from oracle import oracle as orc

    modes = orc.retained_modes(n, n)
    fam = orc.k2_family(orc.Workload(n, n, nz, 4))
    x = orc.flux_inputs(modes, 15, 2 * (nz - 1) // 3, seed)
    t0 = time.perf_counter()
    orc.flux(n, nz, x, family=fam, modes=modes, workers=workers)
    return time.perf_counter() - t0


def cpu_baseline(args):
    workers = os.cpu_count() or 1
    seconds = cpu_flux_once(args.n, args.nz, 129, workers)
    return {"value": 1.0 / seconds, "unit": UNIT, "cores": workers, "kind": "port",
            "sample": f"one 15->4 evaluation of one member at {args.n}x{args.n}, Nz={args.nz} "
                      f"(threaded pocketfft FP64 + BLAS + threaded pointwise; FFTW 3.3.11 is not on this host)"}


def reference_arm(args, dist):
    if dist.rank != 0:
        return None
    workers = os.cpu_count() or 1
    warm = max(0, min(args.warmup, 1))
    for _ in range(warm):
        cpu_flux_once(args.n, args.nz, 129, workers)
    # Bound the timed sample to about two minutes of host work.
    times = []
    budget = 120.0
    for i in range(args.steps):
        times.append(cpu_flux_once(args.n, args.nz, 129 + i, workers))
        if sum(times) > budget:
            break
    sec = statistics.mean(times)
    value = 1.0 / sec
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference modal fixture generator)",
        "config": {"workload": f"15->4 flux {args.n}x{args.n}, Nz={args.nz}, 4 targets, one member per step",
                   "n": args.n, "nz": args.nz, "targets": 4},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                         "sample": f"{len(times)} of {args.steps} steps timed (one evaluation each; "
                                   "FFTW 3.3.11 absent, threaded pocketfft stand-in)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    dist = Dist()
    try:
        if args.impl == "reference":
            line = reference_arm(args, dist)
        elif args.serve:
            line = serve_arm(args, dist)
        elif args.profile_run:
            line = profile_run(args, dist)
        else:
            line = cuda_arm(args, dist)
        if line is not None and dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
