"""The MLP of the learned opening criterion, on the CPU: the oracle's
bfloat16 rounding, its analytic gradient against finite differences, the
budget selection rule, and the shipped trained weights."""
from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import mlp as M


def _random_params(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.TOTAL, np.float32)
    w = M.blocks(p)
    w["W1"][:] = rng.normal(0, 0.5, (8, 32))
    w["b1"][:] = rng.normal(0, 0.1, 32)
    w["W2"][:] = rng.normal(0, 0.25, (32, 32))
    w["b2"][:] = rng.normal(0, 0.1, 32)
    w["W3"][:] = rng.normal(0, 0.2, 32)
    w["b3"][:] = -2.0
    w["mean"][:] = rng.normal(0, 1, 8)
    w["inv_std"][:] = rng.uniform(0.5, 2, 8)
    return p


def test_bf16_rounding():
    vals = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, 1 + 2 ** -8 + 2 ** -20, -2.5, 0.0, 3.0e38], np.float32)
    want = np.array([1.0, 1.0, 1 + 2 ** -6, 1 + 2 ** -7, -2.5, 0.0, np.float32(3.0e38)], np.float32)
    got = M.bf16(vals)
    assert np.array_equal(got[:6], want[:6])
    assert np.all(M.bf16(got) == got)  # idempotent
    assert (got.view(np.uint32) & 0xFFFF == 0).all()
    assert abs(got[6] / want[6] - 1) < 2 ** -8


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = _random_params(1).astype(np.float64)
    X = rng.normal(0, 1.5, (96, 8))
    Y = rng.normal(-2, 0.5, 96)
    g = M.grad_f64(p, X, Y)
    fd = np.zeros(M.TRAINED)
    h = 1e-6
    for i in range(M.TRAINED):
        q = p.copy()
        q[i] += h
        lp = M.loss_f64(q, X, Y)
        q[i] -= 2 * h
        lm = M.loss_f64(q, X, Y)
        fd[i] = (lp - lm) / (2 * h)
    assert np.linalg.norm(g - fd) / np.linalg.norm(fd) < 1e-6


def test_bf16_gradient_close_to_fp64():
    """The BF16 tensor-core gradient is a perturbation of the exact one."""
    rng = np.random.default_rng(4)
    p = _random_params(2)
    X = rng.normal(0, 1.5, (512, 8)).astype(np.float32)
    Y = rng.normal(-2, 0.5, 512).astype(np.float32)
    gb, loss = M.grad_bf16(p, X, Y)
    g64 = M.grad_f64(p.astype(np.float64), X.astype(np.float64), Y.astype(np.float64))
    assert np.linalg.norm(gb - g64) / np.linalg.norm(g64) < 3e-2
    y64, _ = M.forward_f64(p.astype(np.float64), X)
    assert abs(loss / np.sum((y64 - Y) ** 2) - 1) < 3e-2


def test_selection_rule():
    ladder = (2e-4 * 2.0 ** np.arange(8)).astype(np.float32)
    p = np.zeros(M.TOTAL, np.float32)
    w = M.blocks(p)
    w["inv_std"][:] = 1
    # output = log10(alpha) + 1: the error grows with the budget
    w["W1"][0, 0] = 1
    w["b1"][0] = 10
    w["W2"][0, 0] = 1
    w["W3"][0] = 1
    w["b3"][0] = -10 + 1
    feat = np.zeros((5, 7), np.float32)
    # the target lies half a ladder step above the prediction of budget 4
    gp, y = M.select(p, feat, ladder, 10 ** (np.log10(ladder[4]) + 1 + 0.15), 0.9)
    assert np.allclose(y, np.log10(ladder)[None, :] + 1, atol=0.05)
    # the budget is interpolated to where the predicted curve meets the target
    assert np.all(gp[:, 0] == np.float32(0.9))
    assert np.all((gp[:, 1] > ladder[4]) & (gp[:, 1] < ladder[5]))
    assert np.allclose(gp[:, 1], ladder[4] * 10 ** 0.15, rtol=0.15)
    # a target below every prediction takes the most accurate budget
    gp, _ = M.select(p, feat, ladder, 1e-9, 0.9)
    assert np.all(gp[:, 1] == ladder[0])
    # non-finite predictions fall back to the fixed theta 0.5
    w["b3"][0] = np.inf
    gp, _ = M.select(p, feat, ladder, 1e-3, 0.9)
    assert np.all(gp[:, 0] == np.float32(0.5)) and np.all(gp[:, 1] >= 1e30)


def test_shipped_weights():
    from cudagravitydemo_b200 import learned
    if not learned.DEFAULT_WEIGHTS.exists():
        pytest.fail("trained MLP weights are missing (python -m cudagravitydemo_b200.learned)")
    p = learned.load_weights()
    assert p.shape == (M.TOTAL,) and np.all(np.isfinite(p))
    meta = json.loads(learned.DEFAULT_WEIGHTS.with_suffix(".json").read_text())
    # the network explains most of the label variance on held-out snapshots
    assert meta["holdout_mse"] < 0.5 * meta["holdout_mse_of_mean"]
