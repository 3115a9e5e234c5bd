"""Command-line runner: advance a reference-format run directory (or a named synthetic workload)
on the GPU and print one JSON line per time step with the solver statistics.

  python -m si3d_b200.run --workload m1 --steps 3
  python -m si3d_b200.run --run-dir path/to/run --steps 10 --precision mixed

Setting SI3D_LOG_SOLVES=1 also prints, per zeta solve, the iteration count of every inner FP32
solve of iterative refinement (stderr).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m si3d_b200.run")
    src = ap.add_mutually_exclusive_group(required=True)
    src.add_argument("--run-dir")
    src.add_argument("--workload", help="synthetic workload name (c0, c1, c2, t0, t1, m1, p2)")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--precision", choices=["fp64", "mixed", "mg"], default="fp64",
                    help="fp64: plain FP64 MIC-PCG; mixed: FP32 MIC-PCG inside FP64 refinement; "
                         "mg: FP32 multigrid-preconditioned CG inside FP64 refinement")
    ap.add_argument("--itmax", type=int, default=2000)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--ntr", type=int, default=0, help="conservative tracers added to a synthetic workload")
    ap.add_argument("--iturb", type=int, default=0, choices=[0, 1],
                    help="1: a synthetic workload with the Mellor-Yamada 2.5 closure")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the launch shapes of the column stages on the live state first")
    ap.add_argument("--tune", default="",
                    help="apply a launch-shape choice instead: momentum lanes (1 = the fused kernel, 2, 4, 8), "
                         "momentum threads per block, scalar lanes, scalar threads (e.g. 1,128,2,64)")
    args = ap.parse_args(argv)
    tune = tuple(int(v) for v in args.tune.split(",")) if args.tune else None
    if tune is not None and len(tune) != 4:
        ap.error("--tune takes four comma-separated integers")

    from . import build, native, synth
    from .model import GpuRun
    build.build_all()
    run_dir = args.run_dir
    if run_dir is None:
        run_dir = os.path.join(tempfile.gettempdir(), f"si3d_bench_{args.workload}_tr{args.ntr}_t{args.iturb}_r0")
        marker = os.path.join(run_dir, ".complete")
        if not os.path.exists(marker):
            synth.make(args.workload, run_dir, ntr=args.ntr, iturb=args.iturb)
            open(marker, "w").close()
    prec = {"fp64": native.SI3D_FP64, "mixed": native.SI3D_MIXED_IR, "mg": native.SI3D_MIXED_MG}[args.precision]
    run = GpuRun(run_dir, device=args.device, pcg_itmax=args.itmax, precision=prec, autotune=args.autotune)
    try:
        if tune is not None:
            run.set_tune(tune)
        for _ in range(args.steps):
            (s,) = run.run(1)
            print(json.dumps({"step": len(run.stats), "iters": [s.iters[i] for i in range(min(s.nsolves, 24))],
                              "relres": [s.relres[i] for i in range(min(s.nsolves, 24))],
                              "ier": [s.ier[i] for i in range(min(s.nsolves, 24))], "ms": s.ms_total,
                              "ms_pcg": s.ms_pcg}), flush=True)
    finally:
        run.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
