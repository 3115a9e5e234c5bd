"""Ensembles on the GPU: members advanced together by one graph launch per step give exactly the
results (fields bit for bit, iteration counts) of each basin run on its own."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_members(tmp_path_factory):
    from si3d_b200 import ensemble, synth
    root = tmp_path_factory.mktemp("ens")
    ms = ensemble.basins(n=3, seed=11, size_min=(30, 20), size_max=(90, 60), layers=(6, 14))
    ms.append(dataclasses.replace(synth.config("t0"), name="t0"))
    return ensemble.write(ms, str(root))


def test_ensemble_matches_members_run_alone(native_libs, small_members):
    from si3d_b200.ensemble import Ensemble
    from si3d_b200.model import GpuRun
    steps = 6
    ens = Ensemble(small_members)
    try:
        iters, ier, ms = ens.step(steps)
        assert ens.nodes() > 0
        assert (ier == 0).all()
        assert (ms > 0).all()
        got = [(r.get("s").copy(), r.get("uh").copy(), r.get("sal").copy()) for r in ens.runs]
    finally:
        ens.close()
    for k, d in enumerate(small_members):
        run = GpuRun(d, pcg_itmax=2000)
        try:
            st = run.run(steps)
            np.testing.assert_array_equal(run.get("s"), got[k][0])
            np.testing.assert_array_equal(run.get("uh"), got[k][1])
            np.testing.assert_array_equal(run.get("sal"), got[k][2])
            for s in range(1, steps):   # step 1 runs member by member and reports no counts
                ref = [st[s].iters[i] for i in range(st[s].nsolves)]
                assert list(iters[s, k, :len(ref)]) == ref
        finally:
            run.close()


def test_batched_and_member_solves_are_bit_identical(native_libs, small_members):
    """Small members fit the batched launch with the blocks their own solve launches use, so the two
    forms sum every dot product in the same order: fields and iteration counts agree bit for bit."""
    from si3d_b200 import native
    from si3d_b200.ensemble import Ensemble
    out = {}
    for mode in (native.SI3D_ENS_SOLVE_BATCHED, native.SI3D_ENS_SOLVE_MEMBERS):
        ens = Ensemble(small_members)
        try:
            ens.solve_mode(mode)
            iters, ier, _ = ens.step(5)
            assert (ier == 0).all()
            blocks = ens.solve_blocks()
            assert (blocks > 0) == (mode == native.SI3D_ENS_SOLVE_BATCHED)
            out[mode] = (iters, [(r.get("s").copy(), r.get("uh").copy(), r.get("sal").copy()) for r in ens.runs])
        finally:
            ens.close()
    a, b = out[native.SI3D_ENS_SOLVE_BATCHED], out[native.SI3D_ENS_SOLVE_MEMBERS]
    np.testing.assert_array_equal(a[0], b[0])
    for fa, fb in zip(a[1], b[1]):
        for x, y in zip(fa, fb):
            np.testing.assert_array_equal(x, y)


def test_batched_solve_shares_the_grid(native_libs, tmp_path):
    """Members whose own solve launches would need more blocks than the GPU holds share the batched
    launch's blocks: each basin still iterates to its own convergence at the same tolerance, and
    agrees with the basin run alone to rounding (its dot products are summed over fewer blocks)."""
    from si3d_b200 import ensemble, native
    from si3d_b200.ensemble import Ensemble
    from si3d_b200.model import GpuRun
    ms = ensemble.basins(n=4, seed=23, size_min=(480, 380), size_max=(520, 420), layers=(8, 12))
    dirs = ensemble.write(ms, str(tmp_path))
    steps = 4
    ens = Ensemble(dirs)
    try:
        ens.solve_mode(native.SI3D_ENS_SOLVE_BATCHED)
        iters, ier, _ = ens.step(steps)
        assert (ier == 0).all()
        blocks = ens.solve_blocks()
        # each member's own solve launch takes at least ceil((lm / 2) / 1024) blocks of 1024 threads
        # (one node of the larger colour per thread): together more than the batched launch has
        own = [-(-(r.lm // 2) // 1024) for r in ens.runs]
        assert 0 < blocks < sum(own)
        got = [(r.get("s").copy(), r.get("uh").copy()) for r in ens.runs]
    finally:
        ens.close()
    for k, d in enumerate(dirs):
        run = GpuRun(d, pcg_itmax=2000)
        try:
            st = run.run(steps)
            s_ref, u_ref = run.get("s"), run.get("uh")
            assert np.abs(got[k][0] - s_ref).max() <= 1e-10
            assert np.abs(got[k][1] - u_ref).max() <= 1e-9 * max(np.abs(u_ref).max(), 1e-30)
            for s in range(1, steps):
                ref = [st[s].iters[i] for i in range(st[s].nsolves)]
                assert all(abs(int(x) - y) <= 2 for x, y in zip(iters[s, k, :len(ref)], ref))
        finally:
            run.close()


def test_graph_is_captured_once(native_libs, small_members):
    from si3d_b200.ensemble import Ensemble
    ens = Ensemble(small_members[:2])
    try:
        ens.step(2)
        n1 = ens.nodes()
        ens.step(3)
        assert ens.nodes() == n1 > 0
    finally:
        ens.close()


def test_autotune_leaves_the_state_unchanged(native_libs, run_dirs):
    """The autotuner times candidate launch shapes on the live state and restores it: the run that
    continues after tuning is bit-identical to one that never tuned."""
    from si3d_b200.model import GpuRun
    names = ("s", "uh", "vh", "sal", "agx", "ary", "Bth2", "Bth3", "eagx")
    a = GpuRun(run_dirs["t1"], pcg_itmax=2000)
    b = GpuRun(run_dirs["t1"], pcg_itmax=2000)
    try:
        a.run(3)
        b.run(3)
        before = {n: b.get(n).copy() for n in names}
        choice = b.autotune(reps=2)
        assert choice[0] in (1, 2, 4, 8) and choice[1] in (64, 128, 256)
        for n in names:
            np.testing.assert_array_equal(b.get(n), before[n], err_msg=n)
        a.run(3)
        b.run(3)
        for n in names:
            np.testing.assert_array_equal(a.get(n), b.get(n), err_msg=n)
        b.set_tune((2, 64, 4, 256))
        a.run(2)
        b.run(2)
        np.testing.assert_array_equal(a.get("sal"), b.get("sal"))
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("iturb", [0, 1])
def test_fused_momentum_kernel_is_bit_identical(native_libs, tmp_path, iturb):
    """The fused momentum kernel (lanes = 1: explicit terms and column sweep in one pass down each
    face column) against the split cell + column kernels, at every block size: after 6 steps the
    momentum stage's outputs and the model state are bit-identical.  With iturb = 1 the eddy
    viscosity varies from cell to cell, which exercises the carried Av values."""
    from si3d_b200 import synth
    from si3d_b200.model import GpuRun
    d = str(tmp_path / "t1")
    synth.make("t1", d, iturb=iturb)
    names = ("s", "uh", "vh", "sal", "agx", "arx", "agy", "ary", "eagx", "earx", "eagy", "eary", "wp")
    ref = GpuRun(d, pcg_itmax=2000)
    try:
        ref.set_tune((8, 128, 8, 128))
        ref.run(6)
        want = {n: ref.get(n).copy() for n in names}
    finally:
        ref.close()
    for nt in (64, 128, 256):
        g = GpuRun(d, pcg_itmax=2000)
        try:
            g.set_tune((1, nt, 8, 128))
            g.run(6)
            for n in names:
                np.testing.assert_array_equal(g.get(n), want[n], err_msg=f"{n} (threads {nt})")
        finally:
            g.close()
