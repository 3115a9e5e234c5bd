"""CPU oracle of the learned initial guess network (oracle/learn_oracle.cpp): its analytic gradient
against central finite differences (real arithmetic), and the BF16-rounded mode against it."""
import numpy as np
import pytest


def random_params(pyo, seed, scale=0.15):
    rng = np.random.default_rng(seed)
    p = rng.normal(0.0, scale, pyo.net_nparam()).astype(np.float32)
    return p


def random_batch(seed, B=2, H=6, W=7):
    rng = np.random.default_rng(seed)
    feat = rng.normal(0.0, 1.0, (B, H, W, 4)).astype(np.float32)
    mask = (rng.uniform(size=(B, H, W)) > 0.25).astype(np.float32)
    feat[..., 3] = mask
    target = rng.normal(0.0, 1.0, (B, H, W)).astype(np.float32)
    return feat, target, mask


def _offsets():
    stem_b = 9 * 4 * 32
    blk = stem_b + 32
    bsz = 9 * 32 * 32 + 32
    head = blk + 4 * bsz
    return dict(stem_w=(0, stem_b), stem_b=(stem_b, blk), blk_w=(blk, blk + 9 * 32 * 32),
                blk_b=(blk + 9 * 32 * 32, blk + bsz), blk3_w=(blk + 3 * bsz, blk + 3 * bsz + 9 * 32 * 32),
                head_w=(head, head + 288), head_b=(head + 288, head + 289))


def test_gradient_matches_finite_differences(oracle_lib):
    pyo = oracle_lib
    p = random_params(pyo, 1)
    feat, target, mask = random_batch(2)
    loss, g = pyo.net_grad(p, feat, target, mask, bf16=False)
    assert loss > 0
    rng = np.random.default_rng(3)
    checked = 0
    for name, (a, b) in _offsets().items():
        for idx in rng.choice(np.arange(a, b), size=min(6, b - a), replace=False):
            eps = np.float32(1e-4)
            pp = p.copy(); pp[idx] += eps
            pm = p.copy(); pm[idx] -= eps
            step = float(pp[idx]) - float(pm[idx])
            lp, _ = pyo.net_grad(pp, feat, target, mask, bf16=False)
            lm, _ = pyo.net_grad(pm, feat, target, mask, bf16=False)
            fd = (lp - lm) / step
            assert abs(fd - g[idx]) <= 1e-4 * max(abs(fd), abs(g[idx])) + 1e-6, (name, idx, fd, g[idx])
            checked += 1
    assert checked == 37


def test_bf16_mode_is_close_to_real_arithmetic(oracle_lib):
    pyo = oracle_lib
    p = random_params(pyo, 4)
    feat, target, mask = random_batch(5)
    o32 = pyo.net_forward(p, feat, bf16=False)
    o16 = pyo.net_forward(p, feat, bf16=True)
    assert np.abs(o16 - o32).max() <= 5e-2 * np.abs(o32).max()
    _, g32 = pyo.net_grad(p, feat, target, mask, bf16=False)
    _, g16 = pyo.net_grad(p, feat, target, mask, bf16=True)
    cos = float(g16 @ g32 / (np.linalg.norm(g16) * np.linalg.norm(g32)))
    assert cos > 0.99


def test_zero_padding_and_locality(oracle_lib):
    """Outside the image every input reads as zero, and a pixel's output depends only on its
    13 x 13 neighbourhood (6 layers of 3 x 3)."""
    pyo = oracle_lib
    p = random_params(pyo, 6)
    feat, _, _ = random_batch(7, B=1, H=20, W=20)
    base = pyo.net_forward(p, feat, bf16=False)
    f2 = feat.copy()
    f2[0, 0, 0, :] += 1.0
    out = pyo.net_forward(p, f2, bf16=False)
    changed = np.argwhere(np.abs(out - base)[0] > 0)
    assert changed.size > 0
    assert changed[:, 0].max() <= 6 and changed[:, 1].max() <= 6
