"""Run a few RK3 steps of the real-like moist workload for profiling.

    python -m wrf_gpu_b200.profile_step --nx 128 --ny 128 --nz 50 --steps 2

Used as the target command of the ncu captures summarised in ``profiles/``.
"""

from __future__ import annotations

import argparse

import torch

from . import _capi, build, cases, dycore


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=128)
    ap.add_argument("--nz", type=int, default=50)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--periodic", action="store_true")
    ap.add_argument("--diff-6th", type=int, default=0, help="diff_6th_opt of the step (0 off)")
    ap.add_argument("--kernel-times", action="store_true",
                    help="print the last step's per-kernel device time (CUDA events per launch)")
    args = ap.parse_args()
    build.build()
    case = cases.real_like_moist(args.nx, args.ny, args.nz, specified=not args.periodic)
    case.controls["diff_6th_opt"] = args.diff_6th
    nl = dycore.OperationalNamelist.from_case(case)
    stp = dycore.Stepper(nl)
    carry = dycore.carry_from_case(case)
    out = stp.alloc_carry(carry)
    for n in range(args.steps):
        if args.kernel_times and n == args.steps - 1:
            torch.cuda.synchronize()
            _capi.profile_enable(True)
        stp.step_into(carry, out, lead_seconds=0.0)
    torch.cuda.synchronize()
    if args.kernel_times:
        times = _capi.profile_read()
        _capi.profile_enable(False)
        for name, v in times.items():
            print(name, v)
    print("ok", float(out.state.w.abs().max().item()))


if __name__ == "__main__":
    main()
