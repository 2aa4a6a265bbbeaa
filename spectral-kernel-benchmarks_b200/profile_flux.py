"""Run the flux a fixed number of times for a profiler.

    python spectral-kernel-benchmarks_b200/profile_flux.py --n 512 --nz 129 --members 8 --mode fp32 --repeat 2

Executes the device path (no graph) so a kernel profiler sees each launch,
then prints the per-stage event timing of one more evaluation as JSON.
"""

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

import skb_cuda as S  # noqa: E402


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=512)
    p.add_argument("--nz", type=int, default=129)
    p.add_argument("--members", type=int, default=8)
    p.add_argument("--targets", type=int, default=4)
    p.add_argument("--mode", choices=["fp64", "fp32", "tf32x3", "bf16x3"], default="fp32")
    p.add_argument("--repeat", type=int, default=1)
    p.add_argument("--no-profile", action="store_true")
    args = p.parse_args()
    mode = {"fp64": S.FLUX_FP64_PLAIN, "fp32": S.FLUX_FP32, "tf32x3": S.FLUX_SPLIT_TF32X3,
            "bf16x3": S.FLUX_SPLIT_BF16X3}[args.mode]
    flux = S.Flux(args.n, args.nz, targets=args.targets, members=args.members, mode=mode)
    rng = np.random.default_rng(1)
    x = (rng.uniform(-0.125, 0.125, flux.input_elements) + 1j * rng.uniform(-0.125, 0.125, flux.input_elements))
    din = S.DeviceArray.from_numpy(x.astype(flux.device_dtype))
    dout = S.DeviceArray(flux.output_elements * np.dtype(flux.device_dtype).itemsize)
    for _ in range(args.repeat):
        flux.execute_device(din.ptr, dout.ptr)
    S.synchronize()
    if not args.no_profile:
        print(json.dumps(flux.profile(din.ptr, dout.ptr), indent=1))


if __name__ == "__main__":
    main()
