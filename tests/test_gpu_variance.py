"""variance(O, ψ) (statistics.jl:6-22) and EnergyVarianceCorrection
(truncation.jl:269-278, 291-310) on the GPU.

The variance is checked against a restatement of statistics.jl (σ[x⊕ψ] += phase·c
in storage order, Var = Σ|σ|² − σ[ψ]²) and the reference's own known answers
(test_phase1.jl:131-150, test_truncation.jl:305-323).  Under
EnergyVarianceCorrection the sequence evolve! merges unfiltered, measures, applies
the truncation, and measures again (_boundary!, spv_evolve.jl:258-284); it is
checked against the oracle driven through the same steps, with the reference's
own tolerances for the accumulated corrections (test_spv_evolution.jl:95-103)."""
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import filt, heisenberg_gens, rand_terms, strategy

pytestmark = pytest.mark.gpu

NOF = tuple(pp.compile_filter(pp.NoTruncation()))


def variance_ref(terms, ket):
    sigma = {}
    for z, x in sorted(terms):
        c = terms[(z, x)]
        nk = x ^ ket
        sign = bin(z & nk).count("1") % 2
        sp = (4 - bin(z & x).count("1") % 4) % 4
        sigma[nk] = sigma.get(nk, 0) + [1, 1j, -1, -1j][(sp + 2 * sign) % 4] * c
    e2 = sum((v.conjugate() * v).real for v in sigma.values())
    e1 = sigma.get(ket, 0)
    return (e2 - e1 * e1).real


def gpu_from_terms(N, terms):
    ps = pp.PauliSum(N)
    for k, c in terms.items():
        ps[k] = c
    return pp.SparsePauliVector.from_paulisum(ps)


def test_variance_known_answers():
    # test_phase1.jl:131-150: ZI on |00> (eigenstate) has variance 0; XI has variance 1
    for s, expect in (("ZI", 0.0), ("XI", 1.0)):
        b = pp.PauliBasis.from_string(s)
        v = gpu_from_terms(2, {(b.z, b.x): 1.0})
        assert abs(pp.variance(v, 0) - expect) < 1e-12


@pytest.mark.parametrize("N,n", [(8, 300), (40, 5000), (70, 4000), (100, 20000)])
def test_variance_matches_restatement(N, n):
    rng = random.Random(N + n)
    terms = rand_terms(rng, N, n)
    # many terms sharing x words, so sigma entries sum several contributions
    for i, k in enumerate(list(terms)[: n // 2]):
        terms[(k[0], list(terms)[i % 7][1])] = terms.pop(k)
    v = gpu_from_terms(N, terms)
    for ket in (0, rng.getrandbits(N)):
        ref = variance_ref(terms, ket)
        got = pp.variance(v, ket)
        scale = max(1.0, sum(c * c for c in terms.values()))
        assert abs(got - ref) <= 1e-12 * scale, (got, ref)


def test_truncate_energy_variance_correction():
    # test_truncation.jl:305-323
    terms = {}
    for s, c in (("IIII", 1.0), ("ZIII", 0.5), ("XIII", 0.3), ("IIXI", 0.01)):
        b = pp.PauliBasis.from_string(s)
        terms[(b.z, b.x)] = c
    v = gpu_from_terms(4, terms)
    e0, v0 = pp.expectation_value(v, 0), pp.variance(v, 0)
    corr = pp.EnergyVarianceCorrection(0)
    pp.truncate_(v, pp.CoeffTruncation(0.1), corr)
    e1, v1 = pp.expectation_value(v, 0), pp.variance(v, 0)
    assert len(v) == 3
    assert abs(corr.accumulated_energy - (e1 - e0)) < 1e-14
    assert abs(corr.accumulated_variance - (v1 - v0)) < 1e-14
    kept = {k: c for k, c in terms.items() if abs(c) > 0.1}
    assert abs(corr.accumulated_variance - (variance_ref(kept, 0) - variance_ref(terms, 0))) < 1e-12


def oracle_loop(N, terms, gens, angs, ket, apply):
    """The reference's window-1 evolve! under EnergyVarianceCorrection: per rotation,
    rotate and merge unfiltered, measure, truncate, measure."""
    v = orc.OracleSPV(N, 16, 1 << 20)
    v.upload([k[0] for k in terms], [k[1] for k in terms], list(terms.values()))
    acc_e = acc_v = 0.0
    for g, a in zip(gens, angs):
        v.evolve([g], [a], window=1, strict=NOF)
        t = v.terms()
        be, bv = v.expect(ket), variance_ref(t, ket)
        apply(v)
        t = v.terms()
        acc_e += v.expect(ket) - be
        acc_v += variance_ref(t, ket) - bv
    return v, acc_e, acc_v


@pytest.mark.parametrize("adaptive", [False, True])
def test_evolve_energy_variance_correction(adaptive):
    N = 8
    gens, angs = heisenberg_gens(N, dt=0.1, n_trotter=2)
    terms = {(1 << 3, 0): 1.0, ((1 << 1) | (1 << 2), 0): -0.4, (0, 1 << 5): 0.2}
    ket = 0b1010
    if adaptive:
        trunc = pp.AdaptiveTruncation(60, 1e-9)
        apply = lambda v: v.adaptive(60, 1e-9)
    else:
        spec = ("comp", [("coeff", 1e-3), ("weight", 4)])
        trunc = strategy(spec)
        f = filt(spec)
        apply = lambda v: v.compact(f)
    v, acc_e, acc_v = oracle_loop(N, terms, gens, angs, ket, apply)
    g = gpu_from_terms(N, terms)
    g2 = pp.SparsePauliVector(N, 1 << 12, 1 << 20)
    z, x, c = g.to_arrays()
    g2.upload(z, x, c, sorted=True)
    corr = pp.EnergyVarianceCorrection(ket)
    pp.evolve_(g2, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=trunc, correction=corr)
    gz, gx, gc = g2.to_arrays()
    oz, ox, oc = v.arrays()
    assert np.array_equal(gz, oz) and np.array_equal(gx, ox)
    assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64))
    assert abs(acc_e) > 0 and abs(acc_v) > 0
    assert abs(corr.accumulated_energy - acc_e) <= 1e-11 + 1e-9 * abs(acc_e)
    assert abs(corr.accumulated_variance - acc_v) <= 1e-10 + 1e-8 * abs(acc_v)
