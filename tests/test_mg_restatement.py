"""The numpy restatement of the multigrid-mixed zeta solve (oracle/mg_numpy.py) against the FP64
oracle's NSPCG solve of the same system: both stop on test 5 at 1e-12, so their zeta agree to the
tolerance.  This pins the restatement that the GPU multigrid solve is checked against pass by pass."""
import numpy as np
import pytest


def _system(o):
    maps = [o.geti(n) for n in ("l2i", "l2j", "lEC", "lWC", "lNC", "lSC")]
    sx, sy, qq, sp = (o.get(n) for n in ("sx", "sy", "qq", "sp"))
    return maps, sx, sy, qq, sp


@pytest.mark.parametrize("istep", [1, 2])
@pytest.mark.parametrize("name", ["t0", "t1", "c0"])
def test_restatement_matches_nspcg(run_dirs, oracle_lib, name, istep):
    from oracle import mg_numpy
    o = oracle_lib.OracleRun(run_dirs[name], ordering=1, pcg_itmax=2000)
    o.run(2)
    o.stage("momentum", istep)
    o.stage("matcon", istep)
    maps, sx, sy, qq, sp = _system(o)
    z, info = mg_numpy.solve(o.lm, *maps, sx, sy, qq, sp, o.im1, o.jm1)
    assert info["ier"] == 0 and info["stptst"] < 1e-12, info
    assert info["levels"] == mg_numpy.MIN_LEVELS
    # a V-cycle preconditioner: a few inner iterations per refinement pass
    assert info["iters"] <= 15 * info["passes"], info
    o.stage("solve", istep)
    s = o.get("s")[:o.lm]
    assert np.abs(z - s).max() <= 1e-10 * max(np.abs(s).max(), 1e-3)


def test_hierarchy_shapes_and_faces():
    """Coarsening halves rows and columns (rounding up), keeps the total mass and halves the sum of
    the faces that cross between aggregates."""
    from oracle import mg_numpy
    rng = np.random.default_rng(5)
    rows, cols = 13, 10
    m = rng.uniform(0.5, 1.5, (rows, cols)).astype(np.float32)
    fc = rng.uniform(0.0, 4.0, (rows, cols)).astype(np.float32)
    fr = rng.uniform(0.0, 4.0, (rows, cols)).astype(np.float32)
    fc[:, -1] = 0
    fr[-1, :] = 0
    L = mg_numpy.Level(m, fc, fr, (1 / mg_numpy._diag(mg_numpy.Level(m, fc, fr, None))).astype(np.float32))
    G = mg_numpy.coarsen(L)
    assert (G.rows, G.cols) == (7, 5)
    assert abs(float(G.mass.sum(dtype=np.float64)) - float(m.sum(dtype=np.float64))) < 1e-4
    crossing_c = fc[:, 1::2].sum(dtype=np.float64)      # faces from an odd column to the next
    crossing_r = fr[1::2, :].sum(dtype=np.float64)
    assert abs(G.fc.sum(dtype=np.float64) - 0.5 * crossing_c) < 1e-4
    assert abs(G.fr.sum(dtype=np.float64) - 0.5 * crossing_r) < 1e-4
    assert G.fc[:, -1].max() == 0 and G.fr[-1, :].max() == 0
