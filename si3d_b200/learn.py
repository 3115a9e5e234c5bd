"""Learned initial guess for the zeta solve: training data from the plain solver, training with the
project's own forward/backward/Adam kernels (include/si3d_learn.h), parameter files, evaluation.

  python -m si3d_b200.learn train --out si3d_b200/weights/zeta_increment_net.f32
  python -m si3d_b200.learn eval --workload c2 --steps 20

Training examples are recorded by the solver itself (si3d_learn_record): for every zeta solve of a
plain FP64 run it writes the network's four input channels and the target (zeta_solution - sp)/sigma
on the (im1, jm1) image.  Random 64 x 64 crops centred on wet cells form the data set; the network
is fully convolutional, so it is trained on crops and applied to whole basins.  PyTorch only holds
device memory and draws the random crop indices; every network operation is one of the library's
kernels.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import tempfile
import time
from typing import List, Optional

import numpy as np

from . import native

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_PARAMS = os.path.join(HERE, "weights", "zeta_increment_net.f32")
NPARAM = native.NET_NPARAM


# ---------------------------------------------------------------------------- parameters
def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation for the ReLU layers; the residual branches start small and the head
    at zero, so an untrained network predicts a zero increment (the plain guess sp)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    o = 0
    p[o:o + 9 * 4 * 32] = rng.normal(0, np.sqrt(2.0 / (9 * 4)), 9 * 4 * 32)
    o += 9 * 4 * 32 + 32
    for _ in range(4):
        p[o:o + 9 * 32 * 32] = rng.normal(0, 0.1 * np.sqrt(2.0 / (9 * 32)), 9 * 32 * 32)
        o += 9 * 32 * 32 + 32
    return p


def save_params(p: np.ndarray, path: str, meta: Optional[dict] = None) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.asarray(p, dtype="<f4").tofile(path)
    if meta is not None:
        with open(path + ".json", "w") as fh:
            json.dump(meta, fh, indent=1)


def load_params(path: str = DEFAULT_PARAMS) -> np.ndarray:
    p = np.fromfile(path, dtype="<f4")
    if p.size != NPARAM:
        raise ValueError(f"{path}: {p.size} values, expected {NPARAM}")
    return p


# ---------------------------------------------------------------------------- device kernels
class Net:
    """Training-side wrapper of the network kernels on device buffers (torch tensors)."""

    def __init__(self, B: int, H: int, W: int, params: np.ndarray, device: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.g = native.gpu()
        self.B, self.H, self.W = B, H, W
        self.p = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).to(self.dev)
        self.grad = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.t = 0
        nb = self.g.si3d_net_workspace_bytes(B, H, W)
        self.ws = torch.empty(nb, dtype=torch.uint8, device=self.dev)
        self.out = torch.empty((B, H, W), dtype=torch.float32, device=self.dev)
        self.gout = torch.empty_like(self.out)
        self.loss = torch.zeros(native.NET_LOSS_FLOATS, dtype=torch.float32, device=self.dev)

    @staticmethod
    def _ptr(t) -> C.c_void_p:
        return C.c_void_p(t.data_ptr())

    def forward(self, feat):
        assert feat.is_contiguous() and tuple(feat.shape) == (self.B, self.H, self.W, 4)
        native.check(self.g.si3d_net_forward(self._ptr(self.p), self._ptr(feat), self.B, self.H, self.W,
                                             self._ptr(self.out), self._ptr(self.ws), self.ws.numel()))
        return self.out

    def loss_and_grad(self, feat, target, mask) -> None:
        n = self.B * self.H * self.W
        native.check(self.g.si3d_net_loss(self._ptr(self.out), self._ptr(target), self._ptr(mask), n,
                                          self._ptr(self.gout), self._ptr(self.loss)))
        native.check(self.g.si3d_net_backward(self._ptr(self.p), self._ptr(feat), self._ptr(self.gout), self.B, self.H,
                                              self.W, self._ptr(self.grad), self._ptr(self.ws), self.ws.numel()))

    def adam(self, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8) -> None:
        self.t += 1
        native.check(self.g.si3d_net_adam(self._ptr(self.p), self._ptr(self.grad), self._ptr(self.m), self._ptr(self.v),
                                          NPARAM, lr, b1, b2, eps, self.t))

    def params(self) -> np.ndarray:
        return self.p.detach().cpu().numpy().copy()


# ---------------------------------------------------------------------------- data
def record_crops(run_dir: str, steps: int, crops_per_solve: int, crop: int, seed: int, device: int = 0,
                 warmup: int = 3):
    """Run the plain FP64 solver on `run_dir` and return (crops [N][crop][crop][5] on the device,
    solves recorded).  The first `warmup` steps (spin-up from rest) are not recorded."""
    import torch
    from .model import GpuRun
    dev = torch.device("cuda", device)
    run = GpuRun(run_dir, device=device, pcg_itmax=2000)
    g = native.gpu()
    try:
        run.run(warmup)
        hh, ww = C.c_int(0), C.c_int(0)
        nslots = 4
        # one step makes 1 + niter solves (3 with the trapezoidal iterations)
        native.check(g.si3d_learn_record(run.gh, None, 0, C.byref(hh), C.byref(ww)))
        H, W = hh.value, ww.value
        buf = torch.zeros((nslots, H, W, 5), dtype=torch.float32, device=dev)
        native.check(g.si3d_learn_record(run.gh, C.c_void_p(buf.data_ptr()), nslots, C.byref(hh), C.byref(ww)))
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)
        out = []
        wet = None
        half = crop // 2
        for step in range(steps):
            try:
                run.run(1)
            except native.Si3dError as e:   # a basin the plain solver cannot continue: keep what was recorded
                print(f"{run_dir}: stopped at step {warmup + step + 1}: {e}", flush=True)
                break
            native.check(g.si3d_gpu_sync(run.gh))
            n = g.si3d_learn_recorded(run.gh)
            k = min(n, nslots)
            native.check(g.si3d_learn_record(run.gh, C.c_void_p(buf.data_ptr()), nslots, C.byref(hh), C.byref(ww)))
            if wet is None:
                wet = torch.nonzero(buf[0, :, :, 3] > 0)
            for s in range(k):
                pick = wet[torch.randint(0, wet.shape[0], (crops_per_solve,), generator=gen, device=dev)]
                for c in range(crops_per_solve):
                    i0 = int(min(max(int(pick[c, 0]) - half, 0), max(H - crop, 0)))
                    j0 = int(min(max(int(pick[c, 1]) - half, 0), max(W - crop, 0)))
                    out.append(buf[s, i0:i0 + crop, j0:j0 + crop, :].clone())
        native.check(g.si3d_learn_record(run.gh, None, 0, None, None))
        return torch.stack(out), len(out) // crops_per_solve
    finally:
        run.close()


def train(out_path: str, *, basins: int = 6, steps: int = 1111, crops_per_solve: int = 2, crop: int = 64,
          batch: int = 32, iters: int = 4000, lr: float = 1e-3, seed: int = 0, device: int = 0,
          workload: str = "c1", log=print) -> dict:
    """Record ~20k solves of `basins` seeded config-1-style basins, train, save the parameters."""
    import torch
    from . import synth
    from .build import build_all
    build_all()
    torch.cuda.set_device(device)
    dev = torch.device("cuda", device)
    t0 = time.time()
    parts, nsolves = [], 0
    root = tempfile.mkdtemp(prefix="si3d_learn_")
    for k in range(basins):
        d = os.path.join(root, f"{workload}_s{k}")
        synth.make(workload, d, seed_offset=100 + k)
        crops, ns = record_crops(d, steps, crops_per_solve, crop, seed + k, device)
        parts.append(crops)
        nsolves += ns
        log(f"basin {k}: {ns} solves recorded, {crops.shape[0]} crops ({time.time() - t0:.0f} s)")
    val = parts[-1]
    data = torch.cat(parts[:-1]) if len(parts) > 1 else parts[0]
    log(f"training set {tuple(data.shape)}, validation {tuple(val.shape)}")
    net = Net(batch, crop, crop, init_params(seed), device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)

    def batch_of(src, idx):
        b = src[idx]
        return b[..., :4].contiguous(), b[..., 4].contiguous(), b[..., 3].contiguous()

    def val_loss():
        tot, n = 0.0, 0
        for s in range(0, val.shape[0] - batch + 1, batch):
            f, t, m = batch_of(val, torch.arange(s, s + batch, device=dev))
            net.forward(f)
            net.loss_and_grad(f, t, m)
            tot += float(net.loss[0])
            n += 1
        return tot / max(n, 1)

    # loss of the zero prediction (the plain guess sp): mean (target)^2 over wet pixels
    vt, vm = val[..., 4], val[..., 3]
    base = float((vt * vt * vm).sum() / vm.sum())
    log(f"validation loss of the zero increment: {base:.4e}; untrained network: {val_loss():.4e}")
    hist = []
    for it in range(1, iters + 1):
        idx = torch.randint(0, data.shape[0], (batch,), generator=gen, device=dev)
        f, t, m = batch_of(data, idx)
        net.forward(f)
        net.loss_and_grad(f, t, m)
        lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * (it - 1) / iters))
        net.adam(float(lr_t))
        if it % 500 == 0 or it == iters:
            vl = val_loss()
            hist.append((it, float(net.loss[0]), vl))
            log(f"iter {it}: train {float(net.loss[0]):.4e} validation {vl:.4e} ({time.time() - t0:.0f} s)")
    p = net.params()
    meta = dict(workload=workload, basins=basins, steps_per_basin=steps, solves=nsolves, crops=int(data.shape[0]),
                crop=crop, batch=batch, iters=iters, lr=lr, seed=seed, zero_increment_loss=base,
                history=hist, seconds=time.time() - t0)
    save_params(p, out_path, meta)
    log(f"saved {out_path}")
    return meta


# ---------------------------------------------------------------------------- evaluation
def iterations(run_dir: str, steps: int, *, params: Optional[np.ndarray], x0_mode: int, precision: int,
               device: int = 0, warmup: int = 0) -> dict:
    """PCG iterations and zeta after `steps` steps with the given initial guess."""
    from .model import GpuRun
    run = GpuRun(run_dir, device=device, pcg_itmax=2000, x0_mode=x0_mode, precision=precision)
    try:
        if params is not None:
            run.set_net(params)
        st = run.run(warmup + steps)[warmup:]
        its = [s.iters[i] for s in st for i in range(s.nsolves)]
        return dict(iters=its, iters_per_step=sum(its) / steps, max_relres=max(s.relres[i] for s in st
                                                                                 for i in range(s.nsolves)),
                    zeta=run.get("s")[:run.lm].copy(), ms_pcg=sum(s.ms_pcg for s in st) / steps,
                    ms=sum(s.ms_total for s in st) / steps)
    finally:
        run.close()


def time_forward(height: int, width: int, reps: int, params_path: str = DEFAULT_PARAMS) -> int:
    """One inference of the network on a random (1, height, width, 4) feature image, 3 untimed and
    `reps` timed, with CUDA events on the launching stream; prints the mean time per inference."""
    import torch
    from .build import build_all
    build_all()
    net = Net(1, height, width, load_params(params_path))
    feat = torch.randn(1, height, width, 4, device=net.dev)
    for _ in range(3):
        net.forward(feat)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward(feat)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"forward_ms": e0.elapsed_time(e1) / reps, "height": height, "width": width, "reps": reps}))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m si3d_b200.learn")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=DEFAULT_PARAMS)
    t.add_argument("--basins", type=int, default=6)
    t.add_argument("--steps", type=int, default=1111)
    t.add_argument("--iters", type=int, default=4000)
    t.add_argument("--workload", default="c1")
    t.add_argument("--seed", type=int, default=0)
    e = sub.add_parser("eval")
    e.add_argument("--workload", default="c2")
    e.add_argument("--steps", type=int, default=10)
    e.add_argument("--params", default=DEFAULT_PARAMS)
    f = sub.add_parser("forward", help="time one network inference on a (height x width) image")
    f.add_argument("--height", type=int, default=2002)
    f.add_argument("--width", type=int, default=1002)
    f.add_argument("--reps", type=int, default=20)
    f.add_argument("--params", default=DEFAULT_PARAMS)
    args = ap.parse_args(argv)
    if args.cmd == "forward":
        return time_forward(args.height, args.width, args.reps, args.params)
    if args.cmd == "train":
        train(args.out, basins=args.basins, steps=args.steps, iters=args.iters, workload=args.workload, seed=args.seed)
        return 0
    from . import synth
    from .build import build_all
    build_all()
    d = os.path.join(tempfile.gettempdir(), f"si3d_bench_{args.workload}_r0")
    if not os.path.exists(os.path.join(d, ".complete")):
        synth.make(args.workload, d)
        open(os.path.join(d, ".complete"), "w").close()
    p = load_params(args.params)
    res = {}
    for name, x0, prm, prec in [("prev_fp64", native.SI3D_X0_PREV, None, native.SI3D_FP64),
                                ("learned_fp64", native.SI3D_X0_LEARNED, p, native.SI3D_FP64),
                                ("prev_mixed", native.SI3D_X0_PREV, None, native.SI3D_MIXED_IR),
                                ("learned_mixed", native.SI3D_X0_LEARNED, p, native.SI3D_MIXED_IR)]:
        r = iterations(d, args.steps, params=prm, x0_mode=x0, precision=prec)
        res[name] = r
        print(json.dumps({"form": name, "iters_per_step": r["iters_per_step"], "ms": r["ms"], "ms_pcg": r["ms_pcg"],
                          "max_relres": r["max_relres"],
                          "max_dzeta_vs_prev_fp64": float(np.abs(r["zeta"] - res["prev_fp64"]["zeta"]).max())}),
              flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
