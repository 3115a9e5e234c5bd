"""Regenerates the committed fixtures in this folder from the CPU oracle.

The reference ships no golden data for its semi-implicit core, so these fixtures are the oracle's
own outputs on small seeded inputs: they pin the oracle against accidental change (CPU tests) and
let the GPU tests check the CUDA path against stored numbers without running the oracle.

  python tests/golden/make_golden.py        # the small fixtures (seconds)
  python tests/golden/make_golden.py c1     # the 1000-step c1 fixture (about an hour on 6 threads)
"""
import dataclasses
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402
from si3d_b200 import synth  # noqa: E402

STEPS = 10
FIELDS_2D = ("s",)
FIELDS_3D = ("uh", "vh", "sal", "wp")


def run_fixture(name: str, steps: int = STEPS, fields_3d=FIELDS_3D, ntr: int = 0):
    """Oracle state of workload `name` (with `ntr` conservative tracers) after `steps` steps (plain
    FP64, red-black MIC-PCG at test 5, 1e-12) plus the per-solve iteration log."""
    d = os.path.join(tempfile.mkdtemp(), name)
    synth.make(name, d, ntr=ntr)
    o = pyoracle.OracleRun(d, ordering=1, pcg_itmax=2000)
    o.run(steps)
    out = {f: o.get(f)[:o.lm].copy() for f in FIELDS_2D}
    for f in tuple(fields_3d) + tuple(f"tracer{t}" for t in range(1, ntr + 1)):
        out[f] = o.get(f)[:, :o.lm].copy()
    sv = o.solves()
    out["iters"] = np.array([s["iters"] for s in sv], dtype=np.int32)
    out["stptst"] = np.array([s["stptst"] for s in sv])
    out["steps"] = np.int32(steps)
    return out


def pcg_fixture():
    """A seeded SPD 5-point system (SolverSparse's Purdue form) and its oracle solution."""
    sys.path.insert(0, os.path.dirname(HERE))
    from test_oracle_kat import _five_point_system
    coef, jcoef, A = _five_point_system(48, 32, seed=2024)
    b = A @ np.random.default_rng(2025).standard_normal(A.shape[0])
    x0 = np.zeros_like(b)
    x, info = pyoracle.pcg(coef, jcoef, b, x0, pcg_test=5, tol=1e-12, itmax=500, ordering=1)
    return dict(coef=coef, jcoef=jcoef, rhs=b, x=x, iters=np.int32(info["iters"]), stptst=info["stptst"])


C1_STEPS = 1000
C1_SAMPLE_COLUMNS = 2048
C1_SAMPLE_SEED = 1000


def c1_fixture(steps: int = C1_STEPS, threads: int = 6):
    """The 1000 x 500 x 40 workload (seeded random bathymetry and wind stress, dt = 30 s) run for
    `steps` steps by the oracle with the reference's own solver settings apart from the tolerance:
    natural-order MIC-CG, stopping test 5 at 1e-12.  Stored: zeta on every wet column, uh, vh and
    sal at every layer of a seeded sample of wet columns, the per-solve iteration counts and
    stopping values, and max |zeta| after every step (the run's stability record)."""
    os.environ.setdefault("SI3D_ORACLE_THREADS", str(threads))
    d = os.path.join(tempfile.mkdtemp(), "c1")
    b = synth.make("c1", d)
    o = pyoracle.OracleRun(d, ordering=0, pcg_itmax=2000)
    zmax = np.empty(steps)
    for n in range(steps):
        o.run(1)
        zmax[n] = np.abs(o.get("s")[:o.lm]).max()
    cols = np.sort(np.random.default_rng(C1_SAMPLE_SEED).choice(o.lm, C1_SAMPLE_COLUMNS, replace=False))
    out = {"s": o.get("s")[:o.lm].copy(), "columns": cols.astype(np.int32)}
    for f in ("uh", "vh", "sal"):
        out[f] = o.get(f)[:, cols].copy()
        out[f + "_scale"] = np.float64(np.abs(o.get(f)[:, :o.lm]).max())
    sv = o.solves()
    out["iters"] = np.array([s["iters"] for s in sv], dtype=np.int32)
    out["ier"] = np.array([s["ier"] for s in sv], dtype=np.int32)
    out["stptst"] = np.array([s["stptst"] for s in sv])
    out["zeta_max"] = zmax
    out["steps"] = np.int32(steps)
    out["seeds"] = np.array([b.seeds["bathymetry"], b.seeds["wind"]], dtype=np.int64)
    return out


def main():
    pyoracle.build()
    if sys.argv[1:] == ["c1"]:
        np.savez_compressed(os.path.join(HERE, f"c1_oracle_{C1_STEPS}steps.npz"), **c1_fixture())
        return
    np.savez_compressed(os.path.join(HERE, f"t0_oracle_{STEPS}steps.npz"), **run_fixture("t0"))
    np.savez_compressed(os.path.join(HERE, f"t1_oracle_{STEPS}steps.npz"), **run_fixture("t1", fields_3d=()))
    np.savez_compressed(os.path.join(HERE, "pcg_48x32.npz"), **pcg_fixture())
    np.savez_compressed(os.path.join(HERE, f"t0_tracers3_oracle_{STEPS}steps.npz"),
                        **run_fixture("t0", fields_3d=(), ntr=3))


if __name__ == "__main__":
    main()
