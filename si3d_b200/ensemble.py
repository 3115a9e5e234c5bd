"""Ensembles of basins advanced together on one GPU (include/si3d_gpu.h, si3d_ens_*).

The c3 workload: 64 closed basins whose sizes are drawn by seed between 200 x 100 and 1000 x 800
cells, with 20 - 60 layers of 1 m (the depth range of the basin's bathymetry is 2 m to the number of
layers), each with its own seeded Gaussian-random-field bathymetry and land mask (config-1
generators: correlation length 20 cells, 30 % land) and its own smooth wind-stress field whose mean
is drawn in 0.05 - 0.2 Pa (+-50 %), dx = 50 m, dt = 30 s, plain FP64 solver.

Every member keeps its own device state and stream; one ensemble step is one CUDA graph launch.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import native, synth
from .native import check

C3_SEED = 3001


def basins(n: int = 64, seed: int = C3_SEED, size_min=(200, 100), size_max=(1000, 800), layers=(20, 60),
           stress=(0.05, 0.2), dx: float = 50.0, dt: float = 30.0, nsteps: int = 200) -> List[synth.Basin]:
    """The seeded ensemble (member k uses bathymetry seed `seed` * 1000 + 2 k and wind seed + 1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nx = rng.integers(size_min[0], size_max[0] + 1, n)
    ny = rng.integers(size_min[1], size_max[1] + 1, n)
    nl = rng.integers(layers[0], layers[1] + 1, n)
    tau = rng.uniform(stress[0], stress[1], n)
    out = []
    for k in range(n):
        sb, sw = seed * 1000 + 2 * k, seed * 1000 + 2 * k + 1
        depth = synth.random_bathymetry(int(nx[k]), int(ny[k]), sb, corr=20.0, dmin=2.0, dmax=float(nl[k]))
        u = synth.wind_speed_for_stress(synth.stress_field(int(nx[k]), int(ny[k]), sw, mean=float(tau[k]), corr=20.0))
        out.append(synth.Basin(f"e{k:02d}", int(nx[k]), int(ny[k]), dx, dx, depth, int(nl[k]), 1.0, dt, nsteps,
                               dzmin=0.1, uair=u, vair=np.zeros_like(u),
                               seeds={"bathymetry": sb, "wind": sw, "stress_mean": float(tau[k])}))
    return out


def device_bytes(b: synth.Basin) -> int:
    """Device memory of one member: 36 layer-major FP64 fields of (layers + 2) x pitch, plus the
    2-D fields and the zeta system (about 40 FP64 2-D arrays)."""
    lm = int((b.depth > 0).sum())
    pitch = (lm + 1 + 31) // 32 * 32
    return 8 * (36 * (b.nlayers + 2) * pitch + 40 * pitch)


def write(members: Sequence[synth.Basin], root: str) -> List[str]:
    dirs = []
    for b in members:
        d = os.path.join(root, b.name)
        marker = os.path.join(d, ".complete")
        if not os.path.exists(marker):
            synth.write_run(b, d)
            open(marker, "w").close()
        dirs.append(d)
    return dirs


class Ensemble:
    """Members opened from run directories (host set-up + GPU state each) and one si3d_ens handle."""

    def __init__(self, run_dirs: Sequence[str], *, device: int = 0, pcg_itmax: int = 2000, autotune: bool = False):
        from .model import GpuRun
        # each member is autotuned on its own grid before the step graph captures its launch shapes
        self.runs = [GpuRun(d, device=device, pcg_itmax=pcg_itmax, autotune=autotune) for d in run_dirs]
        self.g = native.gpu()
        hs = (C.c_int * len(self.runs))(*[r.gh for r in self.runs])
        e = C.c_int(-1)
        check(self.g.si3d_ens_create(C.cast(hs, C.c_void_p), len(self.runs), C.byref(e)))
        self.e = e.value
        self.n = 0   # steps taken

    def step(self, nsteps: int):
        """Advance every member nsteps; returns (iters, ier, ms) with iters/ier of shape
        [nsteps][members][ENS_MAXSOLVES]."""
        m = len(self.runs)
        iters = np.zeros((nsteps, m, native.ENS_MAXSOLVES), dtype=np.int32)
        ier = np.zeros_like(iters)
        ms = np.zeros(nsteps)
        check(self.g.si3d_ens_step(self.e, self.n + 1, nsteps, native.ptr(iters), native.ptr(ier), native.ptr(ms)))
        self.n += nsteps
        return iters, ier, ms

    def nodes(self) -> int:
        return self.g.si3d_ens_nodes(self.e)

    def solve_mode(self, mode: int) -> None:
        """native.SI3D_ENS_SOLVE_BATCHED (default: each zeta solve of a step is one cooperative launch
        for all members) or native.SI3D_ENS_SOLVE_MEMBERS (one launch per member)."""
        check(self.g.si3d_ens_solve_mode(self.e, mode))

    def solve_blocks(self) -> int:
        """Blocks of the batched solve launch in the captured step (0: per-member form)."""
        return self.g.si3d_ens_solve_blocks(self.e)

    def close(self) -> None:
        if getattr(self, "e", None) is not None:
            self.g.si3d_ens_destroy(self.e)
            self.e = None
        for r in getattr(self, "runs", []):
            r.close()
        self.runs = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
