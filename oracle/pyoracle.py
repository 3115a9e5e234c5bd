"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so) — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker or the timed
CPU stand-in for the reference.  The product package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s"], cwd=HERE, check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, C.c_char_p,
                                 C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_error.restype = C.c_char_p
        L.orc_error.argtypes = [C.c_void_p]
        L.orc_run.argtypes = [C.c_void_p, C.c_int]
        L.orc_dims.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_zlevel.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_set.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_get_int.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_set_int.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.orc_stage.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.orc_nsolves.argtypes = [C.c_void_p]
        L.orc_solve_log.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_pcg.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int,
                              C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double),
                              C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p, C.c_void_p]
        L.orc_trid.argtypes = [C.c_int] + [C.c_void_p] * 5
        L.orc_trid1.argtypes = [C.c_int] + [C.c_void_p] * 3
        L.orc_densty.restype = C.c_double
        L.orc_densty.argtypes = [C.c_double, C.c_double, C.c_double]
        L.orc_net_nparam.restype = C.c_int
        L.orc_net_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_net_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


FIELDS_3D = ("uh uhp uhpp u up upp hu hup hupp ex agx arx vh vhp vhpp v vp vpp hv hvp hvpp agy ary h hp hpp sal salp "
             "salpp rhop Av Dv wp Bth2 Bth3 Bth4 Bex q2 q2p q2pp q2l q2lp q2lpp").split()


class OracleRun:
    """The FP64 restatement of the reference on one run directory."""

    def __init__(self, run_dir: str, *, pcg_test: int = 5, pcg_tol: float = 1e-12, pcg_itmax: int = 200,
                 ordering: int = 1, x0_mode: int = 0, srelpr: float = 2.220446049250313e-16):
        L = lib()
        err = C.create_string_buffer(512)
        h = L.orc_create(run_dir.encode(), pcg_test, pcg_tol, pcg_itmax, ordering, x0_mode, srelpr, err, 512)
        if not h:
            raise RuntimeError(f"oracle: {err.value.decode()}")
        self.h = C.c_void_p(h)
        d = np.zeros(9, dtype=np.int32)
        L.orc_dims(self.h, _p(d))
        self.im1, self.jm1, self.km1, self.lm, self.km, self.k1, self.nts = (int(x) for x in d[:7])
        self.ntr = int(d[8])
        self.lm1 = self.lm + 1

    def run(self, nsteps: int) -> None:
        if lib().orc_run(self.h, nsteps) != 0:
            raise RuntimeError(f"oracle: {lib().orc_error(self.h).decode()}")

    def get(self, name: str) -> np.ndarray:
        if name in FIELDS_3D or name.startswith("tracer"):
            a = np.empty((self.km1, self.lm1), order="F")
        else:
            a = np.empty(self.lm1)
        if lib().orc_get(self.h, name.encode(), _p(a)) < 0:
            raise KeyError(name)
        return a

    def set(self, name: str, value: np.ndarray) -> None:
        a = np.asfortranarray(value, dtype=np.float64)
        if lib().orc_set(self.h, name.encode(), _p(a)) < 0:
            raise KeyError(name)

    def geti(self, name: str) -> np.ndarray:
        a = np.empty(self.lm1, dtype=np.int32)
        if lib().orc_get_int(self.h, name.encode(), _p(a)) < 0:
            raise KeyError(name)
        return a

    def seti(self, name: str, value: np.ndarray) -> None:
        a = np.ascontiguousarray(value, dtype=np.int32)
        if lib().orc_set_int(self.h, name.encode(), _p(a)) < 0:
            raise KeyError(name)

    def stage(self, name: str, istep: int) -> None:
        if lib().orc_stage(self.h, name.encode(), istep) != 0:
            raise RuntimeError(f"oracle: {lib().orc_error(self.h).decode()}")

    def zlevel(self) -> np.ndarray:
        z = np.empty(self.km1)
        lib().orc_zlevel(self.h, _p(z))
        return z

    def solves(self):
        n = lib().orc_nsolves(self.h)
        ints = np.zeros(5 * max(n, 1), dtype=np.int32)
        reals = np.zeros(3 * max(n, 1))
        lib().orc_solve_log(self.h, _p(ints), _p(reals))
        out = []
        for i in range(n):
            out.append(dict(n=int(ints[5 * i]), istep=int(ints[5 * i + 1]), iter=int(ints[5 * i + 2]),
                            iters=int(ints[5 * i + 3]), ier=int(ints[5 * i + 4]), stptst=float(reals[3 * i]),
                            emin=float(reals[3 * i + 1]), emax=float(reals[3 * i + 2])))
        return out

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pcg(coef, jcoef, rhs, x0, *, pcg_test=5, tol=1e-12, itmax=200, ordering=0, srelpr=2.220446049250313e-16):
    """NSPCG mic1 + cg restatement on Purdue arrays (n x 5, column-major, 1-based, 0 = none)."""
    n = rhs.shape[0]
    c = np.asfortranarray(coef, dtype=np.float64)
    j = np.asfortranarray(jcoef, dtype=np.int32)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True)
    it = C.c_int(0)
    st, e0, e1 = C.c_double(0), C.c_double(0), C.c_double(0)
    al = np.zeros(itmax + 2)
    be = np.zeros(itmax + 2)
    ier = lib().orc_pcg(n, _p(c), _p(j), _p(b), _p(x), pcg_test, tol, itmax, ordering, srelpr, C.byref(it), C.byref(st),
                        C.byref(e0), C.byref(e1), _p(al), _p(be))
    return x, dict(iters=it.value, stptst=st.value, emin=e0.value, emax=e1.value, ier=ier,
                   alphas=al[:it.value].copy(), betas=be[:it.value].copy())


def trid(a, b, c, g, r):
    n = len(a)
    # every array handed to the library is bound to a name, so it outlives the call
    aa = np.asfortranarray(np.stack([a, b, c]), dtype=np.float64)
    gc = np.ascontiguousarray(g, dtype=np.float64)
    rc = np.ascontiguousarray(r, dtype=np.float64)
    ag = np.empty(n)
    ar = np.empty(n)
    lib().orc_trid(n, _p(aa), _p(gc), _p(rc), _p(ag), _p(ar))
    return ag, ar


def trid1(a, b, c, d):
    n = len(a)
    aa = np.asfortranarray(np.stack([a, b, c]), dtype=np.float64)
    dc = np.ascontiguousarray(d, dtype=np.float64)
    x = np.empty(n)
    lib().orc_trid1(n, _p(aa), _p(dc), _p(x))
    return x


def densty(t, s, z) -> float:
    return lib().orc_densty(t, s, z)


# ---------------------------------------------------------------------------- learned initial guess
def net_nparam() -> int:
    return lib().orc_net_nparam()


def net_forward(params, feat, *, bf16: bool = True) -> np.ndarray:
    """Network output [B][H][W] for feat [B][H][W][4] (include/si3d_learn.h layout)."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32)
    B, H, W, _ = f.shape
    out = np.empty((B, H, W))
    if lib().orc_net_forward(_p(p), _p(f), B, H, W, int(bf16), _p(out)) != 0:
        raise ValueError("bad shape")
    return out


def net_grad(params, feat, target, mask, *, bf16: bool = True):
    """(loss, d loss / d params) of the masked mean-square error."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    m = np.ascontiguousarray(mask, dtype=np.float32)
    B, H, W, _ = f.shape
    g = np.empty(net_nparam())
    loss = C.c_double(0)
    if lib().orc_net_grad(_p(p), _p(f), _p(t), _p(m), B, H, W, int(bf16), _p(g), C.byref(loss)) != 0:
        raise ValueError("bad shape")
    return loss.value, g
