#!/usr/bin/env python
"""Benchmark of the GPU semi-implicit core on the 2000 x 1000 x 60 workload.

One step = one whole time step of si3d.f90:324-458 (leapfrog fd, settrap, two trapezoidal fd
iterations with settrap2, save): momentum tridiagonals, zeta assembly, three MIC-PCG zeta solves at
relative residual 1e-12, velocities, scalar transport and the time-level bookkeeping, all on one
B200 with the state resident in HBM.  Prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2]

N > 1 (launched under torchrun) runs independent replicas of the basin, one per GPU: the
single-basin path is not sharded (replicas only), so per-GPU work is fixed as N grows.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s/timestep & PCG iters/step at 2000×1000×60: learned+mixed vs plain FP64, same tol"

# Algorithmic bytes (compulsory FP64 streams per unit) of the stages, the frozen byte model:
# 3-D stages count streams per wet 3-D cell N3, 2-D stages per wet column lm, one CG iteration 18
# streams per unknown.
STAGE_STREAMS = {"momentum_x": (14, "N3"), "momentum_y": (14, "N3"), "matcon": (14, "lm"), "pcg_iter": (18, "lm"),
                 "vel": (9, "N3"), "scalar": (16, "N3"), "vel2": (3, "N3"), "settrap": (15, "N3"),
                 "settrap2": (9, "N3"), "save": (15, "N3")}
# One FP32 multigrid-preconditioned CG iteration (the pcg_iter unit of the SI3D_MIXED_MG forms, its
# share of the FP64 refinement passes included in the time): level 0 compulsory streams per wet
# column -- read e, r, p, q, z, the two faces, mass and 1/diag, write e, r, z, p, q -- the coarser
# levels (a third of level 0 together) not counted.
MG_ITER_STREAMS = 15
# The tracer block of one fd call (exTracer + ImTracer for ntr conservative tracers), per wet 3-D
# cell: shared streams read once for all tracers (hup, hvp, uhpp, uh, vhpp, vh, wp, hp, hpp, h,
# Dv, hupp, hvpp) and the three flux arrays written, plus per tracer tracerpp read and tracer
# written.
TRACER_SHARED_STREAMS = 16
TRACER_STREAMS_PER_TRACER = 2
# The Mellor-Yamada 2.5 closure of one fd call, per wet 3-D cell: hp, rhop, up, vp, q2p, q2pp,
# q2lp, q2lpp, Av, Dv read, Av, Dv, q2, q2l written.
STAGE_STREAMS_TURB = 14

WORKLOAD_DESC = {
    "c2": "c2: 2000x1000 cells x 60 layers, seeded random bathymetry and wind stress, dt 30 s, itrap=1 niter=2, "
          "zeta solve to relative residual 1e-12 (test 5)",
}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampler over the timed region."""

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={device}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def traffic_table():
    p = os.path.join(ROOT, "profiles", "traffic_per_launch.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh)
    return {}


def workload_dir(name: str, rank: int, ntr: int = 0, iturb: int = 0) -> str:
    from si3d_b200 import synth
    d = os.path.join(tempfile.gettempdir(), f"si3d_bench_{name}_tr{ntr}_t{iturb}_r{rank}")
    marker = os.path.join(d, ".complete")
    if not os.path.exists(marker):
        synth.make(name, d, ntr=ntr, iturb=iturb)
        open(marker, "w").close()
    return d


def counts(run_dir: str):
    """lm and N3 (wet 3-D cells) of a run directory, from the host set-up."""
    from si3d_b200 import native
    import ctypes as C
    import numpy as np
    h = native.host()
    hm = C.c_int(-1)
    err = C.create_string_buffer(256)
    native.check(h.si3d_host_open(run_dir.encode(), None, C.byref(hm), err, 256))
    dims = (C.c_int * 6)()
    h.si3d_host_dims(hm.value, dims)
    lm = dims[3]
    kmz = np.empty(lm + 1, dtype=np.int32)
    h.si3d_host_get_map(hm.value, b"kmz", native.ptr(kmz))
    h.si3d_host_close(hm.value)
    n3 = int((kmz[:lm] - 1).sum())
    return lm, n3


def physical_cores() -> int:
    """Physical cores among the CPUs this process may run on (one thread per core, hyper-threads
    not counted)."""
    seen = set()
    for c in sorted(os.sched_getaffinity(0)):
        base = f"/sys/devices/system/cpu/cpu{c}/topology/"
        try:
            with open(base + "physical_package_id") as f1, open(base + "core_id") as f2:
                seen.add((f1.read().strip(), f2.read().strip()))
        except OSError:
            seen.add(("cpu", c))
    return max(1, len(seen))


def cpu_port_run(name: str, threads: int, steps: int, warmup: int, ntr: int = 0, iturb: int = 0) -> dict:
    """The CPU restatement of the reference run on the full workload: `warmup` untimed steps, then
    `steps` timed steps.  Natural-order MIC-CG (the reference's ordering), stopping test 5 at 1e-12;
    the column stages on `threads` host threads, the zeta solve serial as the reference runs it on
    OpenMP thread 0 (si3d_procedures.f90:1975-2028).  Only the oracle's library is loaded."""
    import numpy as np
    from oracle import pyoracle
    os.environ["SI3D_ORACLE_THREADS"] = str(threads)   # read once, at the oracle's first column loop
    pyoracle.build()
    d = workload_dir(name, 0, ntr, iturb)
    o = pyoracle.OracleRun(d, ordering=0, pcg_itmax=2000)
    try:
        kmz = o.geti("kmz")
        lm, n3 = o.lm, int((kmz[:o.lm] - 1).sum())
        o.run(max(warmup, 0))
        n0 = len(o.solves())
        t0 = time.perf_counter()
        o.run(steps)
        dt = (time.perf_counter() - t0) / steps
        sv = o.solves()[n0:]
        return {"s_per_step": dt, "lm": lm, "n3": n3, "steps": steps, "warmup": warmup,
                "iters_per_step": sum(s["iters"] for s in sv) / steps}
    finally:
        o.close()


def step_roofline(form: dict, lm: int, n3: int, peak: float, peak_kind: str) -> dict:
    """The whole plain FP64 step against the frozen byte model: per fd call 73 FP64 streams per wet
    cell and 12 per column (3 fd calls per step), per CG iteration 18 streams per unknown, per solve
    4 streams per unknown of set-up (3 solves per step)."""
    alg = 3 * 8 * (73 * n3 + 12 * lm) + 8 * lm * (18 * form["pcg_iters_per_step"] + 3 * 4)
    achieved = alg / form["s_per_step"] / 1e9
    return {"bound": "hbm", "algorithmic_bytes_per_step": alg, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind}


def bench_ensemble(args, ws: int, rank: int, device: int, pg) -> int:
    """c3: the seeded 64-basin ensemble, one CUDA graph launch per step.  With N ranks the members
    are partitioned across the GPUs by size (no collective on the data path); members that do not
    fit the device's free memory are left out and the line says how many ran."""
    import ctypes as C
    import numpy as np
    import torch
    from si3d_b200 import ensemble, native, replicas
    peak, peak_kind = measured_peaks()
    members = ensemble.basins()
    sizes = [ensemble.device_bytes(m) for m in members]
    mine = replicas.partition(sizes, ws)[rank]
    free, _ = torch.cuda.mem_get_info(device)
    budget = 0.9 * free - 2e9
    chosen, used = [], 0
    for i in mine:
        if used + sizes[i] <= budget:
            chosen.append(i)
            used += sizes[i]
    root = os.path.join(tempfile.gettempdir(), "si3d_c3")
    dirs = ensemble.write([members[i] for i in chosen], root)
    lm = [counts(d) for d in dirs]
    t_setup = time.perf_counter()
    ens = ensemble.Ensemble(dirs, device=device, pcg_itmax=args.itmax, autotune=True)
    t_setup = time.perf_counter() - t_setup
    try:
        ens.solve_mode(native.SI3D_ENS_SOLVE_MEMBERS if args.ens_solve == "members" else native.SI3D_ENS_SOLVE_BATCHED)
        ens.step(args.warmup)
        if pg is not None:
            pg.barrier()
        clocks = Clocks(device)
        iters, ier, ms = ens.step(args.steps)
        clk = clocks.stop()
        t = float(ms.sum()) / 1e3 / args.steps
        t = replicas.max_over_ranks(t, pg, device=f"cuda:{device}")
        its = iters.clip(min=0)
        # frozen byte model: per fd 73 streams per wet cell and 12 per column, 18 per column and CG
        # iteration, 4 per column per solve set-up (3 fd and 3 solves per step)
        alg = 0.0
        for k, (lm_k, n3_k) in enumerate(lm):
            alg += 3 * 8 * (73 * n3_k + 12 * lm_k) + 8 * lm_k * (18 * its[:, k, :].sum() / args.steps + 3 * 4)
        achieved = alg / t / 1e9
        line = {
            "metric": "s/timestep of a 64-basin ensemble (one graph launch per step)", "impl": "ours",
            "value": t, "unit": "s/timestep", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "c3: 64 seeded basins 200x100..1000x800 cells, 20-60 layers, 0.05-0.2 Pa, "
                                   "dt 30 s, FP64, zeta solve to 1e-12 (test 5)",
                       "members_run": len(chosen), "members_this_rank": len(mine),
                       "lm": int(sum(a for a, _ in lm)), "n3": int(sum(b for _, b in lm)),
                       "device_gb": used / 1e9, "graph_nodes": ens.nodes(), "setup_s": t_setup,
                       "zeta_solves": ("one cooperative launch for all members per solve, %d blocks" % ens.solve_blocks()
                                       if ens.solve_blocks() > 0 else "one cooperative launch per member and solve")},
            "pcg_iters_per_step_mean_member": float(its.sum() / args.steps / max(len(chosen), 1)),
            "max_ier": int(ier.max()), "min_ier": int(ier.min()),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "whole ensemble step (frozen byte model)",
                         "peak_kind": peak_kind},
            "cpu_baseline": None, "e2e": None, "gpu_launches": 1, "clocks": clk,
        }
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        ens.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--itmax", type=int, default=2000)
    ap.add_argument("--ntr", type=int, default=0,
                    help="conservative tracers carried by the workload (0..30; the headline workload has none)")
    ap.add_argument("--iturb", type=int, default=0, choices=[0, 1],
                    help="1: the Mellor-Yamada 2.5 closure instead of constant eddy coefficients")
    ap.add_argument("--ens-solve", choices=["batched", "members"], default="batched",
                    help="c3: each zeta solve of a step as one launch for all members (batched) or one per member")
    ap.add_argument("--forms", default="",
                    help="comma-separated subset of plain_fp64,mixed_ir,mixed_last,learned_fp64,learned_mixed,"
                         "learned_mg,mg_mixed (the last one is the headline); default: plain_fp64,mixed_ir,mixed_last, "
                         "learned_mixed and learned_mg when trained parameters exist, then mg_mixed")
    args = ap.parse_args()
    ws, rank, local = _dist()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = physical_cores()
        smp = cpu_port_run(args.workload, threads, args.steps, args.warmup, ntr=args.ntr, iturb=args.iturb)
        v = smp["s_per_step"]
        line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "s/timestep", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD_DESC.get(args.workload, args.workload), "form": "plain_fp64",
                           "ntr": args.ntr, "iturb": args.iturb,
                           "lm": smp["lm"], "n3": smp["n3"], "parallelism": "replicas x1",
                           "l2": "host run; no GPU caches involved"},
                "pcg_iters_per_step": smp["iters_per_step"],
                "cpu_baseline": {"value": v, "unit": "s/timestep", "cores": threads, "kind": "port",
                                 "sample": f"the full workload, {smp['warmup']} untimed and {smp['steps']} timed "
                                           f"steps; natural-order MIC-CG (the reference's ordering) at 1e-12; column "
                                           f"stages on {threads} threads (one per physical core), the zeta solve "
                                           f"serial as in the reference"},
                "e2e": {"value": v, "unit": "s/timestep", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import ctypes as C
    import numpy as np
    import torch
    from si3d_b200 import build as sbuild
    from si3d_b200 import native
    from si3d_b200.model import GpuRun

    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)
    sbuild.build_all()
    if args.workload == "c3":
        return bench_ensemble(args, ws, rank, device, pg)
    run_dir = workload_dir(args.workload, rank, args.ntr, args.iturb)
    lm, n3 = counts(run_dir)
    peak, peak_kind = measured_peaks()
    g = native.gpu()

    from si3d_b200 import replicas

    def reduce_max(x):
        return replicas.max_over_ranks(x, pg, device=f"cuda:{device}")

    def measure(form: str, precision: int, x0_mode: int, params, headline: bool) -> dict:
        run = GpuRun(run_dir, device=device, pcg_itmax=args.itmax, precision=precision, x0_mode=x0_mode,
                     autotune=True)
        if params is not None:
            run.set_net(params)
        run.run(args.warmup)

        def barrier():
            torch.cuda.synchronize(device)
            native.check(g.si3d_gpu_sync(run.gh))
            if pg is not None:
                pg.barrier()

        # ------------------------------------------------------------ timed device run
        barrier()
        launches0, _ = run.counters()
        clocks = Clocks(device) if headline else None
        t_wall = time.perf_counter()
        stats = run.run(args.steps)
        barrier()
        t_wall = time.perf_counter() - t_wall
        clk = clocks.stop() if clocks else None
        launches1, _ = run.counters()
        out = {"s_per_step": reduce_max(sum(s.ms_total for s in stats) / 1e3 / args.steps), "launch_shapes": run.tune,
               "pcg_s_per_step": sum(s.ms_pcg for s in stats) / 1e3 / args.steps,
               "pcg_iters_per_step": sum(s.total_iters for s in stats) / args.steps,
               "max_relres": max(max(s.relres[i] for i in range(s.nsolves)) for s in stats),
               "wall_s_per_step": t_wall / args.steps, "gpu_launches": int(launches1 - launches0), "clocks": clk}
        # ------------------------------------------------------------ per-stage profile (2 steps)
        run.profile(True)
        run.run(2)
        _, prof = run.counters()
        run.profile(False)
        stage_ms = {k: v for k, v in prof.items() if v[1] > 0}
        out["stage_ms_per_step"] = {k: v[0] / 2 for k, v in stage_ms.items()}
        out["zeta"] = run.get("s")[:run.lm].copy()   # after warmup + steps + 2 steps, the same in every form
        if "tracer" in stage_ms:
            ms, calls = stage_ms["tracer"]
            alg = 8 * n3 * (TRACER_SHARED_STREAMS + TRACER_STREAMS_PER_TRACER * args.ntr)
            out["tracer_stage"] = {"ntr": args.ntr, "ms_per_call": ms / calls, "calls_per_step": calls / 2,
                                   "ms_per_tracer": ms / calls / args.ntr, "algorithmic_bytes_per_call": alg,
                                   "achieved": alg / (ms / calls * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                                   "frac": alg / (ms / calls * 1e-3) / 1e9 / peak, "peak_kind": peak_kind}
        if "turbulence" in stage_ms:
            ms, calls = stage_ms["turbulence"]
            alg = 8 * n3 * STAGE_STREAMS_TURB
            out["turbulence_stage"] = {"ms_per_call": ms / calls, "calls_per_step": calls / 2,
                                       "algorithmic_bytes_per_call": alg, "achieved": alg / (ms / calls * 1e-3) / 1e9,
                                       "peak": peak, "unit": "GB/s", "frac": alg / (ms / calls * 1e-3) / 1e9 / peak,
                                       "peak_kind": peak_kind}
        dominant = max(stage_ms, key=lambda k: stage_ms[k][0])
        if dominant in ("tracer", "turbulence"):
            ts = out["tracer_stage" if dominant == "tracer" else "turbulence_stage"]
            out["roofline"] = {"bound": "hbm", "achieved": ts["achieved"], "peak": peak, "unit": "GB/s",
                               "frac": ts["frac"], "traffic": None, "kernel": dominant,
                               "algorithmic_bytes_per_call": ts["algorithmic_bytes_per_call"],
                               "ms_per_call": ts["ms_per_call"], "peak_kind": peak_kind}
        elif dominant in STAGE_STREAMS:
            streams, unit = STAGE_STREAMS[dominant]
            if dominant == "pcg_iter" and precision == native.SI3D_MIXED_MG:
                streams = MG_ITER_STREAMS
            units = n3 if unit == "N3" else lm
            word = 4 if (dominant == "pcg_iter" and precision != native.SI3D_FP64) else 8
            per_call_ms = stage_ms[dominant][0] / stage_ms[dominant][1]
            alg_bytes = streams * word * units
            achieved = alg_bytes / (per_call_ms * 1e-3) / 1e9
            tr = traffic_table().get(f"{dominant}:{form}")
            traffic = tr.get("bytes_per_call") if tr and tr.get("workload") == args.workload else None
            out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": achieved / peak, "traffic": traffic, "kernel": dominant,
                               "algorithmic_bytes_per_call": alg_bytes, "ms_per_call": per_call_ms,
                               "peak_kind": peak_kind}
        if headline:
            # -------------------------------------------------------- end to end through the C ABI
            # per step: the surface forcing (uair, vair, cdw) from pinned host memory to the device,
            # one step, zeta back to pinned host memory.  The copies are staged: step n + 1's
            # forcing is copied while step n runs and step n's zeta while step n + 1 runs
            # (si3d_gpu_stage_field / si3d_gpu_fetch_field); every copy is inside the timed region.
            names = ("uair", "vair", "cdw")
            forcing = [{k: torch.from_numpy(run.get(k)).pin_memory() for k in names} for _ in range(2)]
            zeta = [torch.empty(run.lm1, dtype=torch.float64).pin_memory() for _ in range(2)]

            def stage(n):
                for k in names:
                    native.check(g.si3d_gpu_stage_field(run.gh, k.encode(), C.c_void_p(forcing[n % 2][k].data_ptr())))
                native.check(g.si3d_gpu_stage_commit(run.gh))

            def e2e_loop(steps):
                stage(0)
                for n in range(steps):
                    if n + 1 < steps:
                        stage(n + 1)
                    native.check(native.host().si3d_host_run(run.hm, 1, None))
                    native.check(g.si3d_gpu_fetch_field(run.gh, b"s", C.c_void_p(zeta[n % 2].data_ptr())))
                native.check(g.si3d_gpu_copies_wait(run.gh))

            e2e_loop(2)   # warm-up: the staging and snapshot buffers are allocated on first use
            barrier()
            t_e2e = time.perf_counter()
            e2e_loop(args.steps)
            barrier()
            out["e2e"] = {"value": reduce_max((time.perf_counter() - t_e2e) / args.steps), "unit": "s/timestep",
                          "h2d_bytes_per_step": 3 * run.lm1 * 8, "d2h_bytes_per_step": run.lm1 * 8,
                          "copies": "staged: step n + 1's forcing copied during step n, step n's zeta during step n + 1"}
        run.close()
        return out

    from si3d_b200 import learn
    params = learn.load_params() if os.path.exists(learn.DEFAULT_PARAMS) else None
    known = {"plain_fp64": (native.SI3D_FP64, native.SI3D_X0_PREV, None),
             "mixed_ir": (native.SI3D_MIXED_IR, native.SI3D_X0_PREV, None),
             "mixed_last": (native.SI3D_MIXED_IR, native.SI3D_X0_LAST, None),
             "learned_fp64": (native.SI3D_FP64, native.SI3D_X0_LEARNED, params),
             "learned_mixed": (native.SI3D_MIXED_IR, native.SI3D_X0_LEARNED, params),
             "mg_mixed": (native.SI3D_MIXED_MG, native.SI3D_X0_LAST, None),
             "learned_mg": (native.SI3D_MIXED_MG, native.SI3D_X0_LEARNED, params)}
    # the last form is the headline: multigrid inner solves from the latest solution.  The learned
    # guess is measured beside it (same solver, the network's guess for the leapfrog solve); on these
    # basins it saves no multigrid iterations and costs the network's inference, so it is not the headline.
    names = args.forms.split(",") if args.forms else (
        ["plain_fp64", "mixed_ir", "mixed_last"] +
        (["learned_mixed", "learned_mg"] if params is not None else []) + ["mg_mixed"])
    forms = [(f, *known[f]) for f in names]
    if any(f.startswith("learned") for f in names) and params is None:
        raise SystemExit("learned forms need " + learn.DEFAULT_PARAMS)
    res = {}
    for i, (form, prec, x0, prm) in enumerate(forms):
        res[form] = measure(form, prec, x0, prm, headline=(i == len(forms) - 1))
    head_form = forms[-1][0]
    head = res[head_form]
    if "plain_fp64" in res:
        for k, v in res.items():
            v["max_dzeta_vs_plain_fp64_m"] = float(np.abs(v["zeta"] - res["plain_fp64"]["zeta"]).max())

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = physical_cores()
        smp = cpu_port_run(args.workload, threads, steps=2, warmup=1, ntr=args.ntr, iturb=args.iturb)
        v = smp["s_per_step"]
        cpu = {"value": v, "unit": "s/timestep", "cores": threads, "kind": "port",
               "sample": f"the full workload, 1 untimed and 2 timed steps (plain FP64, natural-order MIC-CG at 1e-12, "
                         f"{smp['iters_per_step']:.1f} CG iterations per step); column stages on {threads} threads "
                         f"(one per physical core), the zeta solve serial as in the reference"}

    if rank == 0:
        plain = res.get("plain_fp64", head)
        line = {
            "metric": METRIC, "value": head["s_per_step"], "unit": "s/timestep", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["s_per_step"] * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"plain_fp64": "f64", "mixed_ir": "f64 (fp32 inner solves)", "mixed_last": "f64 (fp32 inner solves)",
                      "learned_fp64": "f64 (bf16 guess net)",
                      "learned_mixed": "f64 (fp32 inner solves, bf16 guess net)",
                      "mg_mixed": "f64 (fp32 multigrid inner solves)",
                      "learned_mg": "f64 (fp32 multigrid inner solves, bf16 guess net)"}[head_form], "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC.get(args.workload, args.workload),
                       "form": head_form, "ntr": args.ntr, "iturb": args.iturb, "lm": lm, "n3": n3, "parallelism": f"replicas x{ws}",
                       "l2": "state (~25 GB) far larger than L2; no flush needed"},
            "pcg_iters_per_step": head["pcg_iters_per_step"], "pcg_s_per_step": head["pcg_s_per_step"],
            "speedup_vs_plain_fp64": plain["s_per_step"] / head["s_per_step"],
            "pcg_speedup_vs_plain_fp64": plain["pcg_s_per_step"] / head["pcg_s_per_step"],
            "forms": {k: {kk: vv for kk, vv in v.items() if kk not in ("clocks", "e2e", "zeta")} for k, v in res.items()},
            "roofline": head.get("roofline"), "cpu_baseline": cpu, "e2e": head["e2e"],
            "plain_step_roofline": step_roofline(plain, lm, n3, peak, peak_kind),
            "gpu_launches": head["gpu_launches"], "clocks": head["clocks"],
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
