"""Learned truncation on the GPU: term features, the tensor-core network's forward
pass and gradient against the CPU restatement (mlp_oracle), training, and the
exact top-budget selection.

Tolerances: the network multiplies bf16 operands with FP32 accumulation on both
sides of the comparison; the restatement accumulates in float64, so outputs agree
to ~1e-5 relative except where an FP32 rounding difference flips a bf16 rounding
of an intermediate (one bf16 ulp, 2^-8 relative, on that element); the bounds
below (5e-3 on outputs, 2e-2 relative Frobenius on each gradient block) leave
room for a few such flips and no more."""
import numpy as np
import pytest

import mlp_oracle as mo
import orc
import pauliprop as pp

pytestmark = pytest.mark.gpu


def lattice_state(layers=3, thresh=1e-5):
    w = pp.circuits.lattice64()
    v = orc.OracleSPV.from_terms(64, w.observable)
    gens = [(p.z, p.x) for p in w.layer]
    f = tuple(pp.compile_filter(pp.CompositeTruncation(pp.CoeffTruncation(thresh), pp.WeightTruncation(12))))
    for _ in range(layers):
        v.evolve(gens, w.angles, window=1, strict=f)
    z, x, c = v.arrays()
    g = pp.SparsePauliVector(64, max(16, 2 * len(c)), max(16, 2 * len(c)))
    g.upload(z, x, c, sorted=True)
    return g, (z, x, c)


def test_features_match_restatement():
    g, (z, x, c) = lattice_state()
    ctx = pp.lattice_feature_ctx(8, 8, 3, 20, 0.3, 0.25, light_cone=(1 << 40) - 1)
    f = pp.features(g, ctx)
    assert f.shape == (len(c), 16)
    rng = np.random.default_rng(0)
    for i in rng.choice(len(c), size=min(400, len(c)), replace=False):
        ref = mo.term_features(ctx, z[i, 0], x[i, 0], c[i])
        assert np.allclose(f[i], ref, rtol=1e-6, atol=1e-6), (i, f[i], ref)


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 5003])
def test_forward_matches_oracle(n):
    rng = np.random.default_rng(n)
    p = mo.init_params(7).astype(np.float32)
    p[mo.NPARAM - 1] = 0.3
    X = rng.normal(0.0, 1.0, (n, 16)).astype(np.float32)
    m = pp.MLP(p)
    y = m.forward(X)
    yr, _ = mo.forward(p.astype(np.float64), X.astype(np.float64))
    err = np.abs(y - yr) / np.maximum(1.0, np.abs(yr))
    assert err.max() <= 5e-3, err.max()
    assert np.median(err) <= 1e-5


@pytest.mark.parametrize("n", [64, 128, 300, 4096])
def test_gradient_matches_oracle(n):
    rng = np.random.default_rng(100 + n)
    p = mo.init_params(3).astype(np.float32)
    X = rng.normal(0.0, 1.0, (n, 16)).astype(np.float32)
    t = rng.normal(0.0, 1.0, n).astype(np.float32)
    m = pp.MLP(p)
    g, loss = m.grad(X, t)
    lr, gr = mo.loss_grad(p.astype(np.float64), X.astype(np.float64), t.astype(np.float64))
    assert abs(loss - lr) <= 1e-4 * max(1.0, abs(lr))
    gd, rd = mo.unpack(g), mo.unpack(gr)
    for name in gd:
        rel = np.linalg.norm(gd[name] - rd[name]) / max(1e-12, np.linalg.norm(rd[name]))
        assert rel <= 2e-2, (name, rel)


def test_training_reduces_loss_and_matches_oracle_step():
    rng = np.random.default_rng(5)
    n = 20000
    X = rng.normal(0.0, 1.0, (n, 16)).astype(np.float32)
    wt = rng.normal(0.0, 0.5, 16)
    t = (np.tanh(X @ wt) + 0.1 * X[:, 0] ** 2).astype(np.float32)
    p0 = mo.init_params(1).astype(np.float32)
    # one full-batch Adam step on the device against the same step in float64
    m = pp.MLP(p0)
    m.load_data(X[:4096], t[:4096])
    m.train(1, batch=4096, lr=1e-3, seed=0)
    p1 = m.get_params()
    _, gr = mo.loss_grad(p0.astype(np.float64), X[:4096].astype(np.float64), t[:4096].astype(np.float64))
    pr, _, _ = mo.adam(p0.astype(np.float64), gr, np.zeros(mo.NPARAM), np.zeros(mo.NPARAM), 1, 1e-3)
    # Adam's first step moves each parameter by ~lr * sign(g): compare the moves
    dev, ref = p1 - p0, pr - p0
    agree = np.mean(np.sign(dev) == np.sign(ref))
    assert agree > 0.97 and np.abs(dev - ref).max() <= 2.1e-3
    # many minibatch steps drive the loss down
    m2 = pp.MLP(p0)
    m2.load_data(X, t)
    losses = m2.train(400, batch=2048, lr=3e-3, seed=1)
    assert losses[-20:].mean() < 0.25 * losses[:5].mean()
    y = m2.forward(X[:2000])
    assert np.mean((y - t[:2000]) ** 2) < 0.3 * np.var(t[:2000])


@pytest.mark.parametrize("budget", [1, 1000, 4321])
def test_learned_truncate_exact_budget(budget):
    g, (z, x, c) = lattice_state()
    n = len(c)
    assert n > budget
    ctx = pp.lattice_feature_ctx(8, 8, 3, 20, 0.3, 0.25)
    p = mo.init_params(11).astype(np.float32)
    m = pp.MLP(p)
    feats = pp.features(g, ctx)
    scores = m.forward(feats)
    keep = mo.budget_select(scores, budget)
    cut = pp.learned_truncate_(g, m, ctx, budget)
    gz, gx, gc = g.to_arrays()
    assert len(gc) == budget
    assert np.array_equal(gz, z[keep]) and np.array_equal(gx, x[keep])
    assert np.array_equal(gc.view(np.uint64), c[keep].view(np.uint64))
    assert cut == scores[keep].min()
    pp.check_spv(g)


def test_learned_truncate_ties_keep_smaller_keys():
    """A network whose output ignores the term (all scores equal) keeps the first
    `budget` terms in key order."""
    g, (z, x, c) = lattice_state()
    ctx = pp.lattice_feature_ctx(8, 8, 3, 20, 0.3, 0.25)
    p = np.zeros(mo.NPARAM, dtype=np.float32)
    p[mo.NPARAM - 1] = 1.5
    m = pp.MLP(p)
    pp.learned_truncate_(g, m, ctx, 777)
    gz, gx, gc = g.to_arrays()
    assert np.array_equal(gz, z[:777]) and np.array_equal(gx, x[:777])
