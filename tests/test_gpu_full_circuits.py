"""The benchmarked circuits end to end: the GPU runs each whole circuit in one
evolve! call from the observable, exactly as bench.py times it (channel after
every Trotter layer, the expectation value returned by the same call), and the
CPU oracle runs it layer by layer as the reference's users do (evolve! of a
layer, then the channel: spv_evolve.jl:312-387, channels.jl:223-243).

Bar: the final surviving key set bit-exact, coefficients bit-identical (window 1:
every output sums at most two separately rounded products) and within
1e-12 * max(1, max|c|) in any case, and <0...0|O|0...0> within
1e-12 * sum_{x=0}|c|.  The 8x8 lattice (3,520 rotations, 6.2e9 term-rotations)
takes the oracle about a minute on one core."""
import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import CHANNEL_KIND, filt, strategy

pytestmark = pytest.mark.gpu


def _spec(w):
    return ("comp", [("coeff", w.thresh)] + ([("weight", w.wmax)] if w.wmax else []))


def _oracle_whole(w):
    f = filt(_spec(w))
    v = orc.OracleSPV.from_terms(w.N, w.observable)
    gens = [(p.z, p.x) for p in w.layer]
    for _ in range(w.layers):
        v.evolve(gens, w.angles, window=1, strict=f)
        if w.channel:
            v.channel(CHANNEL_KIND[w.channel[0]], [w.channel[1]])
    return v


def _gpu_whole(w):
    ps = pp.PauliSum(w.N)
    for z, x, c in w.observable:
        ps[(z, x)] = c
    g = pp.SparsePauliVector.from_paulisum(ps)
    gens, angs = w.generators()
    ch = (w.channel[0], w.channel[1], None) if w.channel else None
    _, e = pp.evolve_(g, gens, angs, truncation=strategy(_spec(w)), channel=ch,
                      channel_every=len(w.layer) if ch else 0, return_expectation=True)
    return g, e


def _check(g, e, v):
    gz, gx, gc = g.to_arrays()
    oz, ox, oc = v.arrays()
    assert gz.shape == oz.shape, (gz.shape, oz.shape)
    assert np.array_equal(gz, oz) and np.array_equal(gx, ox), "final key sets differ"
    assert np.abs(gc - oc).max(initial=0.0) <= 1e-12 * max(1.0, float(np.abs(oc).max(initial=1.0)))
    assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64)), "coefficients not bit-identical"
    diag = np.all(ox == 0, axis=1)
    tol = 1e-12 * max(1e-300, float(np.abs(oc[diag]).sum()))
    assert abs(e - v.expect(0)) <= tol
    assert abs(pp.expectation_value(g, 0) - v.expect(0)) <= tol
    pp.check_spv(g)


def test_config2_lattice64_whole_circuit():
    w = pp.circuits.lattice64()
    g, e = _gpu_whole(w)
    v = _oracle_whole(w)
    _check(g, e, v)
    assert len(v) > 10**6


def test_config3_graph127_whole_circuit():
    w = pp.circuits.random_graph127()
    g, e = _gpu_whole(w)
    v = _oracle_whole(w)
    _check(g, e, v)
    assert len(v) > 10**3
