"""Python API of the GPU semi-implicit core: open a reference-format run directory, run time steps
on the device through the C ABI, read fields back in the reference's (km1, lm1) layout."""
from __future__ import annotations

import ctypes as C
import re
from typing import Optional

import numpy as np

from . import native
from .native import SolverOpts, StepStats, check

FIELDS_3D = ("uh uhp uhpp up upp hu hup hupp agx arx vh vhp vhpp vp vpp hv hvp hvpp agy ary h hp hpp sal salp salpp "
             "rhop Av Dv wp HeatSource Bth2 Bth3 Bth4 q2 q2p q2pp q2l q2lp q2lpp u v").split()
FIELDS_2D = "s sp spp eagx earx eagy eary sx sy dd qq rr uair vair cdw".split()
IFIELDS = ("k1z", "k1u", "k1v")


class GpuRun:
    """One basin on one GPU.  Mirrors the reference's time loop (si3d.f90:324-458)."""

    def __init__(self, run_dir: str, *, device: int = 0, pcg_test: int = 5, pcg_tol: float = 1e-12,
                 pcg_itmax: int = 200, srelpr: float = 2.220446049250313e-16, x0_mode: int = native.SI3D_X0_PREV,
                 precision: int = native.SI3D_FP64, autotune: bool = False, ordering: int = native.SI3D_ORDER_REDBLACK):
        self.h = native.host()
        self.g = native.gpu()
        opts = SolverOpts(pcg_test, pcg_tol, pcg_itmax, srelpr, x0_mode, precision, ordering)
        hm = C.c_int(-1)
        err = C.create_string_buffer(512)
        rc = self.h.si3d_host_open(run_dir.encode(), C.byref(opts), C.byref(hm), err, 512)
        if rc:
            raise native.Si3dError(rc, err.value.decode())
        self.hm = hm.value
        dims = (C.c_int * 6)()
        check(self.h.si3d_host_dims(self.hm, dims))
        self.im1, self.jm1, self.km1, self.lm, self.km, self.nts = list(dims)
        self.lm1 = self.lm + 1
        gh = C.c_int(-1)
        check(self.h.si3d_host_attach_gpu(self.hm, device, C.byref(gh)))
        self.gh = gh.value
        self.stats: list[StepStats] = []
        self.tune: Optional[tuple] = None
        if autotune:
            self.autotune()

    # ------------------------------------------------------------------ stepping
    def run(self, nsteps: int) -> list[StepStats]:
        st = (StepStats * max(nsteps, 1))()
        check(self.h.si3d_host_run(self.hm, nsteps, C.cast(st, C.c_void_p)))
        out = [st[i] for i in range(nsteps)]
        self.stats.extend(out)
        return out

    def stage(self, name: str, istep: int) -> StepStats:
        st = StepStats()
        check(self.g.si3d_gpu_stage(self.gh, name.encode(), istep, C.byref(st)))
        return st

    def profile(self, enable: bool) -> None:
        check(self.g.si3d_gpu_profile(self.gh, 1 if enable else 0))

    def counters(self):
        n = C.c_longlong(0)
        ms = np.zeros(16)
        cnt = np.zeros(16, dtype=np.int64)
        k = check(self.g.si3d_gpu_counters(self.gh, C.byref(n), native.ptr(ms), native.ptr(cnt)))
        return n.value, {native.STAGES[i]: (float(ms[i]), int(cnt[i])) for i in range(k)}

    @property
    def n(self) -> int:
        return self.h.si3d_host_step_count(self.hm)

    # ------------------------------------------------------------------ fields
    def get(self, name: str) -> np.ndarray:
        if name in FIELDS_3D or re.fullmatch(r"tracer(pp)?[0-9]+", name):
            a = np.empty((self.km1, self.lm1), dtype=np.float64, order="F")
        elif name in FIELDS_2D:
            a = np.empty(self.lm1, dtype=np.float64)
        elif name in IFIELDS:
            a = np.empty(self.lm1, dtype=np.int32)
            check(self.g.si3d_gpu_get_ifield(self.gh, name.encode(), native.ptr(a)))
            return a
        else:
            raise KeyError(name)
        check(self.g.si3d_gpu_get_field(self.gh, name.encode(), native.ptr(a)))
        return a

    def set(self, name: str, value: np.ndarray) -> None:
        if name in IFIELDS:
            a = np.ascontiguousarray(value, dtype=np.int32)
            check(self.g.si3d_gpu_set_ifield(self.gh, name.encode(), native.ptr(a)))
            return
        a = np.asfortranarray(value, dtype=np.float64)
        check(self.g.si3d_gpu_set_field(self.gh, name.encode(), native.ptr(a)))

    def map(self, name: str) -> np.ndarray:
        a = np.empty(self.lm1, dtype=np.int32)
        check(self.h.si3d_host_get_map(self.hm, name.encode(), native.ptr(a)))
        return a

    def set_warmstart(self, dz: Optional[np.ndarray]) -> None:
        if dz is None:
            check(self.g.si3d_gpu_set_warmstart(self.gh, None, 0))
            return
        a = np.ascontiguousarray(dz, dtype=np.float64)
        check(self.g.si3d_gpu_set_warmstart(self.gh, native.ptr(a), 0))

    def autotune(self, reps: int = 3) -> tuple:
        """Pick the fastest launch shapes of the column stages on the current state (which is left
        unchanged); returns (momentum lanes, momentum threads, scalar lanes, scalar threads)."""
        ch = np.zeros(4, dtype=np.int32)
        check(self.g.si3d_gpu_autotune(self.gh, reps, native.ptr(ch)))
        self.tune = tuple(int(x) for x in ch)
        return self.tune

    def set_tune(self, choice) -> None:
        ch = np.ascontiguousarray(choice, dtype=np.int32)
        check(self.g.si3d_gpu_set_tune(self.gh, native.ptr(ch)))
        self.tune = tuple(int(x) for x in ch)

    def set_net(self, params: Optional[np.ndarray]) -> None:
        """Load the learned initial guess network (include/si3d_learn.h); None unloads it."""
        if params is None:
            check(self.g.si3d_learn_set_params(self.gh, None))
            return
        a = np.ascontiguousarray(params, dtype=np.float32)
        check(self.g.si3d_learn_set_params(self.gh, native.ptr(a)))

    def close(self) -> None:
        if getattr(self, "hm", None) is not None:
            self.h.si3d_host_close(self.hm)
            self.hm = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_zeta(coef: np.ndarray, jcoef: np.ndarray, rhs: np.ndarray, x0: np.ndarray, *, pcg_test: int = 5,
               tol: float = 1e-12, itmax: int = 200, srelpr: float = 2.220446049250313e-16,
               precision: int = native.SI3D_FP64, ordering: int = native.SI3D_ORDER_REDBLACK):
    """Standalone replacement of the reference's nspcg(mic1, cg, ...) call on Purdue arrays."""
    g = native.gpu()
    lm = rhs.shape[0]
    c = np.asfortranarray(coef, dtype=np.float64)
    j = np.asfortranarray(jcoef, dtype=np.int32)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True)
    it = C.c_int(0)
    st, e0, e1 = C.c_double(0), C.c_double(0), C.c_double(0)
    rc = g.si3d_gpu_solve_zeta(lm, native.ptr(c), native.ptr(j), native.ptr(b), native.ptr(x), pcg_test, tol, itmax,
                               srelpr, precision, ordering, C.byref(it), C.byref(st), C.byref(e0), C.byref(e1))
    check(rc)
    return x, dict(iters=it.value, stptst=st.value, emin=e0.value, emax=e1.value, ier=rc)


def column_tridiag(a, b, c, g, r):
    """Batched trid (two right-hand sides) on the GPU; inputs (n, nsys)."""
    lib = native.gpu()
    n, nsys = a.shape
    arrs = [np.asfortranarray(x, dtype=np.float64) for x in (a, b, c, g, r)]
    ag = np.empty((n, nsys), order="F")
    ar = np.empty((n, nsys), order="F")
    check(lib.si3d_gpu_column_tridiag(n, nsys, *[native.ptr(x) for x in arrs], native.ptr(ag), native.ptr(ar)))
    return ag, ar
