"""AdaptiveTruncation on the GPU against the oracle: the top-k clip
(_apply!(v, ::AdaptiveTruncation), spv_evolve.jl:103-114) alone, and as the
truncation of the sequence evolve! (spv_evolve.jl:312-387), where it is applied
after every unfiltered merge (_boundary!, spv_evolve.jl:258-284).  Bar: key sets
bit-exact, coefficients bit-identical, corrections within 1e-12 relative."""
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import heisenberg_gens, rand_terms

pytestmark = pytest.mark.gpu


def pair(N, terms, **kw):
    v = orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()], **kw)
    z, x, c = v.arrays()
    g = pp.SparsePauliVector(N, max(16, 2 * len(c)), v.append_cap)
    g.upload(z, x, c, sorted=True)
    return g, v


def same(g, v):
    gz, gx, gc = g.to_arrays()
    oz, ox, oc = v.arrays()
    assert np.array_equal(gz, oz) and np.array_equal(gx, ox), "key sets differ"
    assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64)), "coefficients differ"


@pytest.mark.parametrize("N,n,max_terms", [(8, 500, 100), (40, 5000, 4999), (70, 3000, 1), (20, 800, 1000),
                                           (64, 20000, 7777)])
def test_adaptive_clip(N, n, max_terms):
    rng = random.Random(N * 31 + n)
    terms = rand_terms(rng, N, n)
    # ties: many equal magnitudes, both signs
    for i, k in enumerate(list(terms)[: n // 3]):
        terms[k] = (1 if i % 2 else -1) * 0.125 * (1 + i % 4)
    g, v = pair(N, terms)
    pp.truncate_(g, pp.AdaptiveTruncation(max_terms, 1e-3))
    v.adaptive(max_terms, 1e-3)
    same(g, v)
    assert len(g) <= max(max_terms, 0) or len(g) == len(v)


def test_adaptive_zero_budget_and_min_thresh():
    rng = random.Random(3)
    terms = rand_terms(rng, 12, 300)
    g, v = pair(12, terms)
    pp.truncate_(g, pp.AdaptiveTruncation(0, 1e-12))
    v.adaptive(0, 1e-12)
    same(g, v)
    assert len(g) == 0
    g, v = pair(12, terms)
    pp.truncate_(g, pp.AdaptiveTruncation(10_000, 0.2))
    v.adaptive(10_000, 0.2)
    same(g, v)


@pytest.mark.parametrize("window", [1, 3])
def test_evolve_adaptive_matches_oracle(window):
    N = 10
    gens, angs = heisenberg_gens(N, dt=0.1, n_trotter=3)
    g, v = pair(N, {(1 << 4, 0): 1.0, (0, 1 << 2): 0.5})
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, window=window,
               truncation=pp.AdaptiveTruncation(300, 1e-9))
    v.evolve(gens, angs, window=window, adaptive=(300, 1e-9))
    if window == 1:
        same(g, v)
    else:
        # window > 1 sums up to window + 1 values per key; the reference sorts the
        # appends with an unstable quicksort, so equal-key appends may be summed in
        # another order: keys bit-exact, coefficients within 1e-12 relative
        gz, gx, gc = g.to_arrays()
        oz, ox, oc = v.arrays()
        assert np.array_equal(gz, oz) and np.array_equal(gx, ox)
        assert np.abs(gc - oc).max() <= 1e-12 * max(1.0, np.abs(oc).max())
    assert len(g) <= 300


def test_evolve_adaptive_energy_correction():
    N = 9
    gens, angs = heisenberg_gens(N, dt=0.1, n_trotter=2)
    g, v = pair(N, {(1 << 3, 0): 1.0, ((1 << 1) | (1 << 2), 0): -0.4})
    corr = pp.EnergyCorrection(0b101)
    corr.accumulated_energy = 0.25
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=pp.AdaptiveTruncation(120, 1e-9),
               correction=corr)
    e, _ = v.evolve(gens, angs, window=1, adaptive=(120, 1e-9), energy_ket=0b101, energy0=0.25)
    same(g, v)
    assert abs(corr.accumulated_energy - e) <= 1e-12 * max(1.0, abs(e))


def test_evolve_adaptive_with_layer_channel():
    """The layer loop evolve!(v, layer; truncation=Adaptive); channel!(v, p): the
    channel acts after the strategy."""
    w = pp.circuits.chain20(layers=3)
    layer = [(p.z, p.x) for p in w.layer]
    g, v = pair(w.N, {(b[0], b[1]): c for b, c in [((z, x), c) for z, x, c in w.observable]})
    pp.evolve_(g, w.layer * 3, w.angles * 3, truncation=pp.AdaptiveTruncation(2000, 1e-12),
               channel=("depolarizing", 1e-2, None), channel_every=len(layer))
    for _ in range(3):
        v.evolve(layer, w.angles, window=1, adaptive=(2000, 1e-12))
        v.channel(0, [1e-2])
    same(g, v)
