"""Stochastic truncation strategies on the GPU (spv_evolve.jl:35-52, 69-99).

Their random numbers come from a counter-based generator, so parity with the
reference is statistical, as in the reference's own tests (test_stochastic.jl,
test_spv_evolution.jl:169-204): unbiasedness within 5 sigma, promoted
coefficients at +-epsilon, counts and norm preserved; plus the sampler's
inclusion probabilities (|c|^2 / sum |c|^2 for one kept term) and the plumbing of
evolve! (a strategy that cannot fire leaves the deterministic result bit-exact)."""
import math
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import heisenberg_gens, rand_terms

pytestmark = pytest.mark.gpu


def gpu_from_terms(N, terms, cap=None):
    z, x = pp.pack_keys(N, list(terms))
    c = np.array(list(terms.values()), dtype=np.float64)
    v = pp.SparsePauliVector(N, cap or max(16, 2 * len(c)), cap or max(16, 2 * len(c)))
    v.upload(z, x, c, sorted=False)
    return v


def test_stochastic_clip_unbiased_and_promoted():
    N, eps, trials = 6, 0.05, 3000
    terms = {(1, 0): 0.02, (0, 2): -0.01, (4, 4): 0.045, (8, 0): 0.2, (16, 16): -0.7}
    v0 = gpu_from_terms(N, terms)
    z0, x0, c0 = v0.to_arrays()
    keys = [(int(a), int(b)) for a, b in zip(z0[:, 0], x0[:, 0])]
    acc = dict.fromkeys(keys, 0.0)
    rng = random.Random(123)
    for _ in range(trials):
        v = v0.copy()
        pp.stochastic_clip_(v, eps, rng)
        z, x, c = v.to_arrays()
        pp.check_spv(v)
        for a, b, cv in zip(z[:, 0], x[:, 0], c):
            k = (int(a), int(b))
            if abs(terms[k]) < eps:
                assert abs(abs(cv) - eps) < 1e-15 and math.copysign(1, cv) == math.copysign(1, terms[k])
            else:
                assert cv == terms[k]
            acc[k] += cv / trials
    for k, c in terms.items():
        tol = 5 * math.sqrt(eps * abs(c) / trials) + 1e-12
        assert abs(acc[k] - c) < tol, (k, acc[k], c)


def test_stochastic_sampling_smoke_and_norm():
    # test_spv_evolution.jl:169-190
    rng = random.Random(99)
    terms = {}
    while len(terms) < 100:
        terms[(rng.getrandbits(6), rng.getrandbits(6))] = 0.02 * (rng.random() - 0.5)
    v = gpu_from_terms(6, terms)
    n0 = math.sqrt(sum(c * c for c in terms.values()))
    vs = v.copy()
    pp.truncate_(vs, pp.StochasticSamplingTruncation(20, random.Random(1)))
    assert len(vs) == 20
    pp.check_spv(vs)
    _, _, c = vs.to_arrays()
    assert abs(math.sqrt(float(np.sum(c * c))) - n0) <= 1e-10 * n0
    vc = v.copy()
    pp.truncate_(vc, pp.StochasticCoeffTruncation(0.02, random.Random(2)))
    assert len(vc) <= len(v)
    pp.check_spv(vc)
    _, _, c = vc.to_arrays()
    assert np.all(np.abs(c) >= 0.02 - 1e-12)


def test_stochastic_clip_expectation_unbiased():
    # test_spv_evolution.jl:192-204
    rng = random.Random(7)
    terms = {}
    while len(terms) < 100:
        terms[(rng.getrandbits(6), rng.getrandbits(6) if len(terms) % 3 else 0)] = 0.02 * (rng.random() - 0.5)
    v = gpu_from_terms(6, terms)
    ev0 = pp.expectation_value(v, 0)
    acc, M = 0.0, 400
    r = random.Random(3)
    for _ in range(M):
        vt = v.copy()
        pp.stochastic_clip_(vt, 0.02, r)
        acc += pp.expectation_value(vt, 0)
    assert abs(acc / M - ev0) < 0.02


def test_sampling_inclusion_probabilities():
    """One kept term: term i is kept with probability |c_i|^2 / sum |c|^2 and its
    coefficient scaled to keep the norm."""
    terms = {(1, 0): 1.0, (2, 0): -math.sqrt(2.0), (4, 0): math.sqrt(3.0), (8, 0): 2.0}
    w = {k: c * c for k, c in terms.items()}
    tot = sum(w.values())
    v0 = gpu_from_terms(5, terms)
    counts = dict.fromkeys(terms, 0)
    trials = 4000
    rng = random.Random(11)
    for _ in range(trials):
        v = v0.copy()
        pp.truncate_(v, pp.StochasticSamplingTruncation(1, rng))
        z, x, c = v.to_arrays()
        k = (int(z[0, 0]), int(x[0, 0]))
        counts[k] += 1
        assert abs(abs(c[0]) - math.sqrt(tot)) <= 1e-12 * math.sqrt(tot)
        assert math.copysign(1, c[0]) == math.copysign(1, terms[k])
    for k in terms:
        p = w[k] / tot
        assert abs(counts[k] / trials - p) < 5 * math.sqrt(p * (1 - p) / trials) + 1e-3, (k, counts[k], p)


@pytest.mark.parametrize("strategy", ["sample", "clip"])
def test_evolve_stochastic_plumbing(strategy):
    """A stochastic strategy that cannot fire (n_keep above every count; epsilon 0)
    leaves the sequence evolve! equal, bit for bit, to the untruncated run."""
    N = 8
    gens, angs = heisenberg_gens(N, dt=0.1, n_trotter=2)
    terms = {(1 << 3, 0): 1.0, (0, 1 << 2): 0.5}
    v = orc.OracleSPV(N, 16, 1 << 20)
    v.upload([k[0] for k in terms], [k[1] for k in terms], list(terms.values()))
    v.evolve(gens, angs, window=1)
    g = gpu_from_terms(N, terms, cap=1 << 12)
    s = (pp.StochasticSamplingTruncation(1 << 40, random.Random(5)) if strategy == "sample"
         else pp.StochasticCoeffTruncation(0.0, random.Random(5)))
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=s)
    gz, gx, gc = g.to_arrays()
    oz, ox, oc = v.arrays()
    assert np.array_equal(gz, oz) and np.array_equal(gx, ox)
    assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64))


def test_evolve_stochastic_sampling_bounds_terms():
    N = 10
    gens, angs = heisenberg_gens(N, dt=0.1, n_trotter=2)
    g = gpu_from_terms(N, {(1 << 4, 0): 1.0}, cap=1 << 12)
    n_ref = g.copy()
    pp.evolve_(n_ref, [pp.PauliBasis(N, a, b) for a, b in gens], angs)
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs,
               truncation=pp.StochasticSamplingTruncation(40, random.Random(8)))
    assert len(n_ref) > 40 and len(g) <= 40
    pp.check_spv(g)
