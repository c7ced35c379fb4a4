"""Learned correction of the compressed path's preconditioner (no counterpart in the
reference; the plain method is precond.c:138-391).

CPU: the numpy MLP of oracle/mlp_oracle.py against finite differences.
GPU: the library's forward, gradient and Adam kernels against that oracle; the training
targets against a known answer (one leaf: the corrected block is the block itself); the
A/B of GMRES iterations with and without the trained network on a held-out structure at
the same tolerance, with Z unchanged; the fall back to the plain preconditioner.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402


def _data(n, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, mo.IN)).astype(np.float32)
    t = (0.3 * np.tanh(x[:, :2] @ np.array([[1.0, -0.5], [0.3, 0.8]])) +
         0.05 * rng.normal(size=(n, 2))).astype(np.float32)
    return x, t


def _init(seed=0):
    rng = np.random.default_rng(seed)
    parts = []
    for fin, fout in ((mo.IN, mo.H), (mo.H, mo.H), (mo.H, mo.OUT)):
        parts.append(rng.uniform(-1, 1, fout * fin) / np.sqrt(fin))
        parts.append(rng.uniform(-0.1, 0.1, fout))
    return np.concatenate(parts).astype(np.float32)


def test_oracle_gradient_matches_finite_differences():
    w = _init().astype(np.float64)
    x, t = _data(9)
    _, g = mo.loss_grad(w, x, t)
    rng = np.random.default_rng(3)
    idx = rng.choice(mo.NPARAM, 40, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(mo.NPARAM)
        e[i] = h
        fd = (mo.loss_only(w + e, x, t) - mo.loss_only(w - e, x, t)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-8 + 1e-6 * abs(g[i]), (i, fd, g[i])


def test_oracle_adam_fits():
    x, t = _data(64)
    _, hist = mo.adam(_init(), x, t, 200, 3e-3)
    assert hist[-1] < 0.2 * hist[0]


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 37, 1000])
def test_forward_matches_oracle(n):
    from openpeec_b200 import api
    assert api.mlp_nparam() == mo.NPARAM
    w = _init()
    x, _ = _data(n)
    y = api.mlp_predict(w, x)
    yo, _ = mo.forward(w, x)
    assert np.abs(y - yo).max() <= 1e-5 * (1 + np.abs(yo).max())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [5, 33, 1000])
def test_gradient_matches_oracle(n):
    """GPU backward pass (per-CTA partial gradients, fixed-order reduction) against the
    float64 oracle on the same float32 weights: FP32 accumulation bar 1e-5 (norm)."""
    from openpeec_b200 import api
    w = _init()
    x, t = _data(n)
    loss, g = api.mlp_grad(w, x, t)
    lo, go = mo.loss_grad(w, x, t)
    assert abs(loss - lo) <= 1e-5 * lo
    assert np.linalg.norm(g - go) <= 1e-5 * np.linalg.norm(go)
    # deterministic: the same call gives the same bits
    _, g2 = api.mlp_grad(w, x, t)
    assert np.array_equal(g, g2)


@pytest.mark.gpu
def test_adam_matches_oracle():
    """pb_mlp_train (GPU Adam) follows the float64 Adam of the oracle step by step."""
    from openpeec_b200 import api
    w = _init()
    x, t = _data(200)
    w_gpu, hist = api.mlp_train(w, x, t, steps=30, lr=1e-3, want_loss=True)
    w_cpu, hist_cpu = mo.adam(w, x, t, 30, 1e-3)
    assert np.all(np.abs(hist - hist_cpu) <= 1e-4 * hist_cpu), (hist[:5], hist_cpu[:5])
    assert np.abs(w_gpu - w_cpu).max() <= 1e-2


@pytest.mark.gpu
def test_samples_single_leaf_known_answer():
    """A structure of at most 32 current cells is one leaf: the leaf block is the whole
    block, S_r = A_LL, and every target is 0."""
    from openpeec_b200 import api, configs, geometry
    prob = geometry.build(geometry.parse_peec(configs.cfg4(3, 3, 1, 2)))
    assert len(prob.seg) <= 32
    with api.Context(prob) as ctx:
        for f in (1e6, 2e9):
            x, t = ctx.pc_samples(f)
            assert np.all(np.isfinite(x))
            assert np.abs(t).max() <= 1e-6, np.abs(t).max()


@pytest.mark.gpu
def test_learned_preconditioner_ab():
    """Train on seeded bar stacks of the family (data from the plain method), then solve a
    held-out 20 x 12 x 4 stack with and without the trained network at the same GMRES
    tolerance. The answer must not change (both solves reach the 1e-10 relative residual);
    the iteration counts are what the network gains or costs, and they are printed."""
    from openpeec_b200 import api, configs, geometry, pc_learn
    fam = pc_learn.plate_family(seed=0, count=4, grid=(6, 12))
    X, T = pc_learn.collect([p for _, p in fam])
    assert np.all(np.isfinite(X)) and np.all(np.isfinite(T))
    w, hist = pc_learn.train(X, T, steps=1500, want_loss=True)
    assert hist[-1] < 0.6 * T.var(0).mean(), (hist[-1], T.var(0))  # explains most of the variance
    prob = geometry.build(geometry.parse_peec(configs.cfg4(20, 12, 4, 2)))
    rows = []
    with api.Context(prob) as ctx:
        for f in (1e6, 1e9):
            z0, s0 = ctx.sweep([f], compress=1)
            z1, s1 = ctx.sweep([f], compress=1, pc_mlp=w)
            assert np.abs(z1 - z0).max() <= 1e-8 * np.abs(z0).max()
            rows.append((f, s0["gmres_its_max"], s1["gmres_its_max"], s1["pc_mlp_fallbacks"]))
    print("learned preconditioner A/B (f, plain its, learned its, fallbacks):", rows)


@pytest.mark.gpu
def test_non_finite_prediction_falls_back():
    from openpeec_b200 import api, configs, geometry
    prob = geometry.build(geometry.parse_peec(configs.cfg4(8, 8, 2, 2)))
    w = np.zeros(mo.NPARAM, np.float32)
    w[-2] = np.nan
    with api.Context(prob) as ctx:
        z0, s0 = ctx.sweep([1e6, 1e9], compress=1)
        z1, s1 = ctx.sweep([1e6, 1e9], compress=1, pc_mlp=w)
    assert s1["pc_mlp_fallbacks"] == 2
    assert s1["gmres_its_max"] == s0["gmres_its_max"]
    assert np.array_equal(z0, z1)


@pytest.mark.gpu
def test_exact_leaf_blocks_do_not_halve_iterations():
    """The negative evidence behind the learned leaf-block correction, as an experiment
    anyone can rerun (pb_sweep_opts.pc_exact_leaf): every leaf block of the Lp kernel block
    replaced by the exact S_r = ((A_LL^-1)_rr)^-1, the best any correction of the leaf
    blocks alone (learned or not) can give the block-diagonal + Schur preconditioner. On
    the held-out 20 x 12 x 4 bar stack the iteration count stays within a few of the plain
    preconditioner's, far from 2x fewer: the count is set by the far-field coupling of
    divergence-free currents, which no leaf block reaches (the two-level preconditioner,
    pc_coarse, is what removes it). The answer is unchanged."""
    from openpeec_b200 import api, configs, geometry
    prob = geometry.build(geometry.parse_peec(configs.cfg4(20, 12, 4, 2)))
    rows = []
    with api.Context(prob) as ctx:
        for f in (1e6, 1e9):
            z0, s0 = ctx.sweep([f], compress=1)
            z1, s1 = ctx.sweep([f], compress=1, pc_exact_leaf=1)
            z2, s2 = ctx.sweep([f], compress=1, pc_coarse=1)
            assert np.abs(z1 - z0).max() <= 1e-8 * np.abs(z0).max()
            rows.append((f, s0["gmres_its_max"], s1["gmres_its_max"], s2["gmres_its_max"]))
    print("GMRES iterations (f, plain, exact leaf blocks, two-level):", rows)
    for f, plain, exact, coarse in rows:
        assert 2 * exact > plain            # exact leaf blocks: not 2x fewer
        assert coarse < plain               # the coarse space does reduce them
