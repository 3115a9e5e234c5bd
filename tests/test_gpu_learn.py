"""Learned initial guess on the GPU: the network kernels against the CPU oracle
(oracle/learn_oracle.cpp, BF16 rounding points emulated), the solver-side recorder, and the
effect of the network on the zeta solve."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _groups():
    sb = 9 * 4 * 32
    blk = sb + 32
    bsz = 9 * 32 * 32 + 32
    head = blk + 4 * bsz
    g = {"stem": (0, blk)}
    for k in range(4):
        g[f"block{k}"] = (blk + k * bsz, blk + (k + 1) * bsz)
    g["head"] = (head, head + 289)
    return g


def _case(seed, B=2, H=19, W=37, scale=0.15):
    rng = np.random.default_rng(seed)
    from si3d_b200 import native
    p = rng.normal(0.0, scale, native.NET_NPARAM).astype(np.float32)
    feat = rng.normal(0.0, 1.0, (B, H, W, 4)).astype(np.float32)
    mask = (rng.uniform(size=(B, H, W)) > 0.3).astype(np.float32)
    feat[..., 3] = mask
    target = rng.normal(0.0, 1.0, (B, H, W)).astype(np.float32)
    return p, feat, target, mask


def _gpu_net(native_libs, p, feat, target, mask):
    import torch
    from si3d_b200.learn import Net
    B, H, W, _ = feat.shape
    net = Net(B, H, W, p)
    dev = net.dev
    f = torch.from_numpy(feat).to(dev).contiguous()
    t = torch.from_numpy(target).to(dev).contiguous()
    m = torch.from_numpy(mask).to(dev).contiguous()
    out = net.forward(f).cpu().numpy().copy()
    net.loss_and_grad(f, t, m)
    return out, float(net.loss[0].cpu()), net.grad.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("shape", [(2, 19, 37), (1, 8, 16), (3, 5, 3)])
def test_forward_matches_oracle(native_libs, oracle_lib, shape):
    B, H, W = shape
    p, feat, target, mask = _case(11, B, H, W)
    out, _, _ = _gpu_net(native_libs, p, feat, target, mask)
    ref = oracle_lib.net_forward(p, feat, bf16=True)
    scale = np.abs(ref).max()
    assert np.abs(out - ref).max() <= 2e-2 * scale
    assert np.sqrt(np.mean((out - ref) ** 2)) <= 2e-3 * scale


def test_gradients_match_oracle(native_libs, oracle_lib):
    """Every parameter group's gradient from the GPU backward kernels against the CPU oracle with
    the same BF16 rounding points."""
    p, feat, target, mask = _case(12)
    out, loss, g = _gpu_net(native_libs, p, feat, target, mask)
    loss_ref, g_ref = oracle_lib.net_grad(p, feat, target, mask, bf16=True)
    assert loss == pytest.approx(loss_ref, rel=2e-2)
    for name, (a, b) in _groups().items():
        num = np.linalg.norm(g[a:b] - g_ref[a:b])
        den = np.linalg.norm(g_ref[a:b])
        assert num <= 3e-2 * den, (name, num / den)


def test_adam_step(native_libs):
    import torch
    from si3d_b200 import native
    g = native.gpu()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    p0 = rng.normal(size=1000).astype(np.float32)
    gr = rng.normal(size=1000).astype(np.float32)
    p, grad = torch.from_numpy(p0.copy()).to(dev), torch.from_numpy(gr).to(dev)
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    for t in (1, 2):
        native.check(g.si3d_net_adam(C.c_void_p(p.data_ptr()), C.c_void_p(grad.data_ptr()), C.c_void_p(m.data_ptr()),
                                     C.c_void_p(v.data_ptr()), 1000, 1e-2, 0.9, 0.999, 1e-8, t))
    mm = 0.1 * gr
    vv = 0.001 * gr * gr
    q = p0 - 1e-2 * (mm / 0.1) / (np.sqrt(vv / 0.001) + 1e-8)
    mm = 0.9 * mm + 0.1 * gr
    vv = 0.999 * vv + 0.001 * gr * gr
    q = q - 1e-2 * (mm / (1 - 0.81)) / (np.sqrt(vv / (1 - 0.999 ** 2)) + 1e-8)
    np.testing.assert_allclose(p.cpu().numpy(), q, rtol=1e-5, atol=1e-6)


def test_recorder_writes_features_and_target(native_libs, run_dirs, oracle_lib):
    """The solver's recorder: one image per solve; mask and depth channels match the grid; the
    residual channel is normalised by its own rms (mean of c0^2 over wet cells is 1); land is zero."""
    import torch
    from si3d_b200 import native
    from si3d_b200.model import GpuRun
    run = GpuRun(run_dirs["t1"], pcg_itmax=2000)
    g = native.gpu()
    try:
        run.run(3)
        hh, ww = C.c_int(0), C.c_int(0)
        native.check(g.si3d_learn_record(run.gh, None, 0, C.byref(hh), C.byref(ww)))
        H, W = hh.value, ww.value
        buf = torch.zeros((4, H, W, 5), dtype=torch.float32, device="cuda")
        native.check(g.si3d_learn_record(run.gh, C.c_void_p(buf.data_ptr()), 4, C.byref(hh), C.byref(ww)))
        run.run(1)
        native.check(g.si3d_gpu_sync(run.gh))
        n = g.si3d_learn_recorded(run.gh)
        assert n == 3
        rec = buf.cpu().numpy()
        native.check(g.si3d_learn_record(run.gh, None, 0, None, None))
        l2i, l2j = run.map("l2i")[:run.lm] - 1, run.map("l2j")[:run.lm] - 1
        o = oracle_lib.OracleRun(run_dirs["t1"], ordering=1, pcg_itmax=2000)
        hhs = o.get("hhs")[:o.lm]
        wet = np.zeros((H, W), dtype=bool)
        wet[l2i, l2j] = True
        for k in range(n):
            img = rec[k]
            np.testing.assert_array_equal(img[l2i, l2j, 3], np.ones(run.lm, dtype=np.float32))
            np.testing.assert_allclose(img[l2i, l2j, 2], (hhs / 30.0).astype(np.float32), rtol=1e-6)
            assert np.all(img[~wet] == 0.0)
            c0 = img[l2i, l2j, 0].astype(np.float64)
            assert np.mean(c0 * c0) == pytest.approx(1.0, rel=1e-5)
            assert np.all(np.isfinite(img)) and np.abs(img[l2i, l2j, 4]).max() > 0
        assert rec[3].max() == 0.0 and rec[3].min() == 0.0   # slot 3 unused
    finally:
        run.close()


def test_untrained_network_is_the_plain_guess(native_libs, run_dirs):
    """The initialisation zeroes the head, so before training the learned guess is sp on the leapfrog
    solves (where sp is the latest solution) and the latest solution on the others: the solves are
    those of x0 = SI3D_X0_LAST, iteration for iteration."""
    from si3d_b200 import native
    from si3d_b200.learn import init_params, iterations
    d = run_dirs["t1"]
    a = iterations(d, 4, params=None, x0_mode=native.SI3D_X0_LAST, precision=native.SI3D_FP64)
    b = iterations(d, 4, params=init_params(0), x0_mode=native.SI3D_X0_LEARNED, precision=native.SI3D_FP64)
    assert a["iters"] == b["iters"]
    assert np.abs(a["zeta"] - b["zeta"]).max() <= 1e-12


def test_untrained_network_with_multigrid_solves(native_libs, run_dirs):
    """The learned guess feeds the multigrid-mixed solve as well: an untrained network reproduces the
    x0 = SI3D_X0_LAST multigrid run iteration for iteration, at the unchanged tolerance."""
    from si3d_b200 import native
    from si3d_b200.learn import init_params, iterations
    d = run_dirs["t1"]
    a = iterations(d, 4, params=None, x0_mode=native.SI3D_X0_LAST, precision=native.SI3D_MIXED_MG)
    b = iterations(d, 4, params=init_params(0), x0_mode=native.SI3D_X0_LEARNED, precision=native.SI3D_MIXED_MG)
    assert a["iters"] == b["iters"]
    assert b["max_relres"] < 1e-12
    assert np.abs(a["zeta"] - b["zeta"]).max() <= 1e-12


PARAMS = os.path.join(ROOT, "si3d_b200", "weights", "zeta_increment_net.f32")


@pytest.fixture(scope="module")
def unseen_c1(tmp_path_factory):
    """A basin of the training family (1000 x 500 x 40, seeded random bathymetry and wind) with seeds
    the network was not trained on."""
    from si3d_b200 import synth
    d = str(tmp_path_factory.mktemp("unseen") / "c1")
    synth.make("c1", d, seed_offset=57)
    return d


@pytest.mark.skipif(not os.path.exists(PARAMS), reason="no trained parameters committed")
@pytest.mark.parametrize("precision", ["fp64", "mg"])
def test_trained_network_against_latest_solution(native_libs, unseen_c1, precision):
    """Ablation against the method without the network.  With the network loaded the leapfrog solve
    of each step starts from sp + the predicted increment and the trapezoidal solves from the latest
    solution, so the method without it is x0 = SI3D_X0_LAST: the trapezoidal solves are identical and
    only the leapfrog solves can gain.  On a basin the network was not trained on, 6 steps after 2
    of warm-up: the leapfrog solves take fewer iterations in total (FP64 MIC-CG) or no more (the
    multigrid inner solves, which need about a dozen), every solve reaches relative residual 1e-12 and
    the accepted zeta agrees to 1e-8 m."""
    from si3d_b200 import native
    from si3d_b200.learn import iterations, load_params
    prec = native.SI3D_FP64 if precision == "fp64" else native.SI3D_MIXED_MG
    last = iterations(unseen_c1, 6, params=None, x0_mode=native.SI3D_X0_LAST, precision=prec, warmup=2)
    learned = iterations(unseen_c1, 6, params=load_params(PARAMS), x0_mode=native.SI3D_X0_LEARNED, precision=prec,
                         warmup=2)
    assert learned["max_relres"] < 1e-12 and last["max_relres"] < 1e-12
    lf_last, lf_learned = sum(last["iters"][0::3]), sum(learned["iters"][0::3])
    print(f"leapfrog iterations over 6 steps: latest solution {lf_last}, learned {lf_learned}; "
          f"per step {last['ms']:.3f} / {learned['ms']:.3f} ms")
    if precision == "fp64":
        assert lf_learned < lf_last
    else:
        assert lf_learned <= lf_last
    assert np.abs(learned["zeta"] - last["zeta"]).max() <= 1e-8


@pytest.mark.skipif(not os.path.exists(PARAMS), reason="no trained parameters committed")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_trained_network_reduces_iterations(native_libs, run_dirs, precision):
    """The trained network against the reference's own guess (x0 = sp for every solve) on a small
    basin it was not trained on: fewer CG iterations (most of the gain comes from the trapezoidal
    solves starting at the latest solution; the ablation against that is the test above), and the
    accepted solution agrees with the plain one to 1e-8 m (both meet relative residual 1e-12)."""
    from si3d_b200 import native
    from si3d_b200.learn import iterations, load_params
    prec = native.SI3D_FP64 if precision == "fp64" else native.SI3D_MIXED_IR
    d = run_dirs["t1"]
    plain = iterations(d, 8, params=None, x0_mode=native.SI3D_X0_PREV, precision=prec, warmup=2)
    learned = iterations(d, 8, params=load_params(PARAMS), x0_mode=native.SI3D_X0_LEARNED, precision=prec, warmup=2)
    assert learned["max_relres"] < 1e-12 and plain["max_relres"] < 1e-12
    assert sum(learned["iters"]) < sum(plain["iters"])
    assert np.abs(learned["zeta"] - plain["zeta"]).max() <= 1e-8
