"""ctypes bindings of the two in-tree native libraries (include/si3d_gpu.h, include/si3d_host.h).

Loading fails loudly: there is no Python or CPU fallback for any stage.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBDIR = os.path.join(_HERE, "_lib")

SI3D_FP64 = 0
SI3D_MIXED_IR = 1
SI3D_MIXED_MG = 2
SI3D_ORDER_REDBLACK = 1
SI3D_ORDER_NATURAL = 2
SI3D_X0_PREV, SI3D_X0_ZERO, SI3D_X0_LEARNED, SI3D_X0_LAST, SI3D_X0_HIST = 0, 1, 2, 3, 4


class Si3dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"si3d error {code}: {msg}")
        self.code = code


SI3D_OUT_PTRACK, SI3D_OUT_TRACER, SI3D_OUT_PLANE = 1, 2, 3


class Grid(C.Structure):
    _fields_ = [("im1", C.c_int), ("jm1", C.c_int), ("km1", C.c_int), ("k1", C.c_int), ("lm", C.c_int),
                ("l2i", C.POINTER(C.c_int)), ("l2j", C.POINTER(C.c_int)), ("lEC", C.POINTER(C.c_int)),
                ("lWC", C.POINTER(C.c_int)), ("lNC", C.POINTER(C.c_int)), ("lSC", C.POINTER(C.c_int)),
                ("kmz", C.POINTER(C.c_int)), ("hhs", C.POINTER(C.c_double)), ("hhu", C.POINTER(C.c_double)),
                ("hhv", C.POINTER(C.c_double)), ("zlevel", C.POINTER(C.c_double))]


class Params(C.Structure):
    _fields_ = [("dt", C.c_double), ("dx", C.c_double), ("dy", C.c_double), ("Av0", C.c_double),
                ("Dv0", C.c_double), ("Ax0", C.c_double), ("Ay0", C.c_double), ("f", C.c_double),
                ("theta", C.c_double), ("cd", C.c_double), ("cw", C.c_double), ("beta", C.c_double),
                ("iadv", C.c_int), ("itrmom", C.c_int), ("ihd", C.c_int), ("ibc", C.c_int), ("isal", C.c_int),
                ("itrap", C.c_int), ("niter", C.c_int), ("ismooth", C.c_int), ("pcg_test", C.c_int),
                ("pcg_tol", C.c_double), ("pcg_itmax", C.c_int), ("srelpr", C.c_double), ("ordering", C.c_int),
                ("x0_mode", C.c_int), ("precision", C.c_int), ("ntr", C.c_int), ("iturb", C.c_int)]


class StepStats(C.Structure):
    _fields_ = [("nsolves", C.c_int), ("iters", C.c_int * 24), ("relres", C.c_double * 24), ("ier", C.c_int * 24),
                ("total_iters", C.c_int), ("ms_total", C.c_double), ("ms_pcg", C.c_double)]


class SolverOpts(C.Structure):
    _fields_ = [("pcg_test", C.c_int), ("pcg_tol", C.c_double), ("pcg_itmax", C.c_int), ("srelpr", C.c_double),
                ("x0_mode", C.c_int), ("precision", C.c_int), ("ordering", C.c_int)]


GPU_SYMBOLS = {
    "si3d_gpu_init": (C.c_int, [C.POINTER(Grid), C.POINTER(Params), C.c_int, C.POINTER(C.c_int)]),
    "si3d_gpu_set_field": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_get_field": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_set_field_f32": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_get_field_f32": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_set_ifield": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_get_ifield": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_density": (C.c_int, [C.c_int]),
    "si3d_gpu_fd": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(StepStats)]),
    "si3d_gpu_stage": (C.c_int, [C.c_int, C.c_char_p, C.c_int, C.POINTER(StepStats)]),
    "si3d_gpu_settrap": (C.c_int, [C.c_int]),
    "si3d_gpu_settrap2": (C.c_int, [C.c_int]),
    "si3d_gpu_save": (C.c_int, [C.c_int, C.c_int]),
    "si3d_gpu_step": (C.c_int, [C.c_int, C.c_int, C.POINTER(StepStats)]),
    "si3d_gpu_set_warmstart": (C.c_int, [C.c_int, C.c_void_p, C.c_int]),
    "si3d_gpu_solve_zeta": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                      C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "si3d_gpu_column_tridiag": (C.c_int, [C.c_int, C.c_int] + [C.c_void_p] * 7),
    "si3d_gpu_column_tridiag_noalloc": (C.c_int, [C.c_int, C.c_int] + [C.c_void_p] * 8),
    "si3d_gpu_profile": (C.c_int, [C.c_int, C.c_int]),
    "si3d_gpu_counters": (C.c_int, [C.c_int, C.POINTER(C.c_longlong), C.c_void_p, C.c_void_p]),
    "si3d_gpu_output_frame": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_longlong,
                                        C.POINTER(C.c_longlong)]),
    "si3d_gpu_output_frame_async": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_longlong,
                                              C.POINTER(C.c_longlong), C.POINTER(C.c_ulonglong)]),
    "si3d_gpu_output_wait": (C.c_int, [C.c_int, C.c_ulonglong]),
    "si3d_gpu_host_alloc": (C.c_int, [C.c_longlong, C.POINTER(C.c_void_p)]),
    "si3d_gpu_host_free": (C.c_int, [C.c_void_p]),
    "si3d_gpu_sync": (C.c_int, [C.c_int]),
    "si3d_gpu_test_wait_limit": (C.c_int, [C.c_int, C.c_longlong, C.c_int]),
    "si3d_gpu_set_open_boundaries": (C.c_int, [C.c_int, C.c_int] + [C.c_void_p] * 6 + [C.c_double, C.c_int,
                                                                                       C.c_void_p, C.c_void_p]),
    "si3d_gpu_strerror": (C.c_char_p, [C.c_int]),
    "si3d_gpu_finalize": (None, [C.c_int]),
    "si3d_gpu_autotune": (C.c_int, [C.c_int, C.c_int, C.c_void_p]),
    "si3d_gpu_set_tune": (C.c_int, [C.c_int, C.c_void_p]),
    "si3d_ens_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "si3d_ens_step": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "si3d_ens_nodes": (C.c_int, [C.c_int]),
    "si3d_gpu_stage_field": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_stage_commit": (C.c_int, [C.c_int]),
    "si3d_gpu_fetch_field": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_gpu_copies_wait": (C.c_int, [C.c_int]),
    "si3d_ens_solve_mode": (C.c_int, [C.c_int, C.c_int]),
    "si3d_ens_solve_blocks": (C.c_int, [C.c_int]),
    "si3d_ens_destroy": (None, [C.c_int]),
    # learned initial guess (include/si3d_learn.h)
    "si3d_learn_set_params": (C.c_int, [C.c_int, C.c_void_p]),
    "si3d_learn_record": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "si3d_learn_recorded": (C.c_int, [C.c_int]),
    "si3d_net_workspace_bytes": (C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    "si3d_net_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_size_t]),
    "si3d_net_loss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "si3d_net_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_size_t]),
    "si3d_net_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_float,
                                C.c_float, C.c_float, C.c_int]),
    "si3d_net_sync": (C.c_int, []),
}
ENS_MAXSOLVES = 4
SI3D_ENS_SOLVE_MEMBERS = 0
SI3D_ENS_SOLVE_BATCHED = 1
NET_NPARAM = 9 * 4 * 32 + 32 + 4 * (9 * 32 * 32 + 32) + 9 * 32 + 1
NET_LOSS_FLOATS = 2 + 2 * 148

HOST_SYMBOLS = {
    "si3d_host_open": (C.c_int, [C.c_char_p, C.POINTER(SolverOpts), C.POINTER(C.c_int), C.c_char_p, C.c_int]),
    "si3d_host_dims": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "si3d_host_get_map": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p]),
    "si3d_host_get_zlevel": (C.c_int, [C.c_int, C.c_void_p]),
    "si3d_host_attach_gpu": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "si3d_host_run": (C.c_int, [C.c_int, C.c_int, C.c_void_p]),
    "si3d_host_step_count": (C.c_int, [C.c_int]),
    "si3d_host_close": (None, [C.c_int]),
}

STAGES = ("momentum_x", "momentum_y", "matcon", "pcg_setup", "pcg_iter", "pcg_finish", "slayer_h", "vel",
          "scalar", "vel2", "settrap", "settrap2", "save", "learn", "tracer", "turbulence")

_gpu = None
_host = None


def _bind(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def gpu_lib_path() -> str:
    return os.path.join(_LIBDIR, "libsi3d_gpu.so")


def host_lib_path() -> str:
    return os.path.join(_LIBDIR, "libsi3d_host.so")


def gpu():
    """The CUDA core.  Raises if the library has not been built."""
    global _gpu
    if _gpu is None:
        p = gpu_lib_path()
        if not os.path.exists(p):
            raise RuntimeError(f"{p} is missing: build it with `python -m si3d_b200.build`")
        _gpu = _bind(C.CDLL(p, mode=C.RTLD_GLOBAL), GPU_SYMBOLS)
    return _gpu


def host():
    global _host
    if _host is None:
        gpu()
        p = host_lib_path()
        if not os.path.exists(p):
            raise RuntimeError(f"{p} is missing: build it with `python -m si3d_b200.build`")
        _host = _bind(C.CDLL(p), HOST_SYMBOLS)
    return _host


def check(rc: int) -> int:
    if rc < 0:
        raise Si3dError(rc, gpu().si3d_gpu_strerror(rc).decode())
    return rc


def ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)
