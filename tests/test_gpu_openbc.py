"""Open boundaries with a specified water-surface elevation on the GPU against the oracle.

Two basins in the reference's input format (si3d_b200/synth.py): t2, a channel forced by a tide
through its west end, and t3, a basin with open east, north and south sides.  30 whole time steps
through the C ABI on both sides (the boundary series read from openbcNN.txt, openbc0's sp, the
stage adjustments of openbcUVH, MODexmom4openBCX/Y, MODqqddrr4openBC, MODvel4openBC and openbcSCA):
zeta within 1e-9 m, velocities within 1e-8 and temperature within 1e-10 of the field's scale, the
boundary cells on the series value, iteration counts within two of the oracle's in the same ordering.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def obc_dirs(tmp_path_factory):
    from si3d_b200 import synth
    base = tmp_path_factory.mktemp("obc_runs")
    out = {}
    for name in ("t2", "t3"):
        d = str(base / name)
        synth.make(name, d)
        out[name] = d
    return out


@pytest.mark.parametrize("name", ["t2", "t3"])
@pytest.mark.parametrize("form", ["FP64", "NATURAL", "MIXED_MG"])
def test_open_boundary_steps_match_oracle(native_libs, oracle_lib, obc_dirs, name, form):
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    steps = 30
    ordering = 0 if form == "NATURAL" else 1
    o = oracle_lib.OracleRun(obc_dirs[name], ordering=ordering, pcg_itmax=2000)
    o.run(steps)
    kw = dict(pcg_itmax=2000)
    if form == "NATURAL":
        kw["ordering"] = native.SI3D_ORDER_NATURAL
    if form == "MIXED_MG":
        kw["precision"] = native.SI3D_MIXED_MG
        kw["x0_mode"] = native.SI3D_X0_LAST
    g = GpuRun(obc_dirs[name], **kw)
    try:
        st = g.run(steps)
        assert all(s.ier[i] == 0 for s in st for i in range(s.nsolves))
        assert np.abs(g.get("s") - o.get("s")).max() <= 1e-9
        for f, tol in (("uh", 1e-8), ("vh", 1e-8), ("wp", 1e-7), ("sal", 1e-10), ("h", 1e-10)):
            a = o.get(f)
            err = np.abs(g.get(f) - a).max() / max(np.abs(a).max(), 1e-300)
            assert err <= tol, f"{name}/{form}:{f} rel err {err:.3e}"
        if form != "MIXED_MG":
            it_o = [s["iters"] for s in o.solves()]
            it_g = [s.iters[i] for s in st for i in range(s.nsolves)]
            assert len(it_o) == len(it_g)
            assert max(abs(a - b) for a, b in zip(it_o, it_g)) <= 2, (it_o[:9], it_g[:9])
    finally:
        g.close()


def test_open_boundaries_refuse_fp32_mic(native_libs, obc_dirs):
    """The FP32 MIC inner solves of SI3D_MIXED_IR are not built for open boundaries: refused."""
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    with pytest.raises(native.Si3dError):
        GpuRun(obc_dirs["t2"], precision=native.SI3D_MIXED_IR)
