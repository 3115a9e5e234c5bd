"""The bounded device waits run out, on purpose, and the handle stays usable.

Every grid-barrier wait of the cooperative zeta solves gives up after a bounded number of polls and
the solve returns SI3D_ETIMEOUT instead of hanging.  Here a test hook makes one solve's barriers wait
for a block that does not exist, with a limit of 10^4 polls: the fd call must come back with
SI3D_ETIMEOUT through the C ABI, and after the state is put back the same handle must advance
exactly as a handle that never timed out.  Nothing faults: every block leaves its loop once the
limit is reached or another block has given up.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE_3D = ("uh uhp uhpp up upp hu hup hupp agx arx vh vhp vhpp vp vpp hv hvp hvpp agy ary h hp hpp sal salp salpp "
            "rhop Av Dv wp HeatSource Bth2 Bth3 Bth4").split()
STATE_2D = "s sp spp eagx earx eagy eary sx sy dd qq rr uair vair cdw".split()
STATE_I = ("k1z", "k1u", "k1v")


@pytest.mark.parametrize("precision", ["FP64", "MIXED_IR", "MIXED_MG"])
def test_barrier_wait_runs_out_and_handle_recovers(native_libs, run_dirs, precision):
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    prec = getattr(native, f"SI3D_{precision}")
    g = native.gpu()
    a = GpuRun(run_dirs["t1"], pcg_itmax=2000, precision=prec)
    b = GpuRun(run_dirs["t1"], pcg_itmax=2000, precision=prec)
    try:
        a.run(2)
        b.run(2)
        snap = {f: a.get(f) for f in STATE_3D + STATE_2D + list(STATE_I)}
        assert g.si3d_gpu_test_wait_limit(a.gh, 0, 1) == -101          # out-of-range arguments refused
        assert g.si3d_gpu_test_wait_limit(a.gh, 10_000, 1) == 0
        st = native.StepStats()
        rc = g.si3d_gpu_fd(a.gh, 3, 1, 0, C.byref(st))
        assert rc == -105, g.si3d_gpu_strerror(rc).decode()              # SI3D_ETIMEOUT
        assert native.check(g.si3d_gpu_sync(a.gh)) == 0                  # the context still answers
        for f, v in snap.items():
            a.set(f, v)
        sa = a.run(2)
        sb = b.run(2)
        assert [s.iters[i] for s in sa for i in range(s.nsolves)] == [s.iters[i] for s in sb for i in range(s.nsolves)]
        for f in ("s", "uh", "vh", "sal"):
            np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)
    finally:
        a.close()
        b.close()
