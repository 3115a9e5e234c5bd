"""Staged inputs and asynchronous reads (si3d_gpu_stage_field / stage_commit / fetch_field /
copies_wait): a loop that stages step n + 1's surface forcing while step n runs, and reads each
step's zeta back on a copy stream, advances exactly as the loop that copies synchronously."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned(native, n):
    """A pinned host array of n doubles (si3d_gpu_host_alloc keeps it for the process)."""
    p = C.c_void_p()
    native.check(native.gpu().si3d_gpu_host_alloc(8 * n, C.byref(p)))
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n,))


def test_staged_forcing_and_fetched_zeta_match_synchronous_copies(native_libs, run_dirs):
    from si3d_b200.model import GpuRun
    native = native_libs
    g = native.gpu()
    steps = 6
    a = GpuRun(run_dirs["t1"], pcg_itmax=2000)
    b = GpuRun(run_dirs["t1"], pcg_itmax=2000)
    try:
        base = {k: a.get(k).copy() for k in ("uair", "vair", "cdw")}
        scale = {"uair": lambda n: 1.0 + 0.05 * n, "vair": lambda n: 1.0 - 0.03 * n, "cdw": lambda n: 1.0}

        def forcing(n):
            return {k: base[k] * scale[k](n) for k in base}

        zeta_sync = []
        for n in range(steps):
            for k, v in forcing(n).items():
                a.set(k, v)
            a.run(1)
            zeta_sync.append(a.get("s").copy())

        lm1 = b.lm1
        staged = [{k: _pinned(native, lm1) for k in base} for _ in range(steps)]
        zeta = [_pinned(native, lm1) for _ in range(steps)]
        for n in range(steps):
            for k, v in forcing(n).items():
                staged[n][k][:] = v

        def stage(n):
            for k in base:
                native.check(g.si3d_gpu_stage_field(b.gh, k.encode(), staged[n][k].ctypes.data_as(C.c_void_p)))
            native.check(g.si3d_gpu_stage_commit(b.gh))

        stage(0)
        for n in range(steps):
            if n + 1 < steps:
                stage(n + 1)   # copied while step n runs
            b.run(1)
            native.check(g.si3d_gpu_fetch_field(b.gh, b"s", zeta[n].ctypes.data_as(C.c_void_p)))
        native.check(g.si3d_gpu_copies_wait(b.gh))
        for n in range(steps):
            np.testing.assert_array_equal(zeta[n], zeta_sync[n])
        for k in ("s", "uh", "vh", "sal", "uair"):
            np.testing.assert_array_equal(b.get(k), a.get(k))
    finally:
        a.close()
        b.close()


def test_stage_refuses_a_third_waiting_group(native_libs, run_dirs):
    from si3d_b200.model import GpuRun
    native = native_libs
    g = native.gpu()
    run = GpuRun(run_dirs["t0"], pcg_itmax=2000)
    try:
        buf = _pinned(native, run.lm1)
        buf[:] = run.get("uair")
        for _ in range(2):
            native.check(g.si3d_gpu_stage_field(run.gh, b"uair", buf.ctypes.data_as(C.c_void_p)))
            native.check(g.si3d_gpu_stage_commit(run.gh))
        assert g.si3d_gpu_stage_field(run.gh, b"uair", buf.ctypes.data_as(C.c_void_p)) == -101   # SI3D_EDIMS
        assert g.si3d_gpu_stage_field(run.gh, b"zeta_unknown", buf.ctypes.data_as(C.c_void_p)) == -103   # SI3D_ENAME
        run.run(2)   # each step takes one group
        native.check(g.si3d_gpu_copies_wait(run.gh))
        np.testing.assert_array_equal(run.get("uair"), buf)
    finally:
        run.close()
