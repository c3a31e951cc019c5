"""Pins the CPU oracle (a restatement of the SPV engine) against an independent
restatement of the reference's Dict path — the A/B parity the reference's own
tests use (test_spv_evolution.jl:33-167, test_spv_equivalence.jl:138-159)."""
import math
import random

import pytest

import dictpath
import orc
from helpers import filt, heisenberg_gens, maxdiff, rand_terms

STRATS = [("none",), ("coeff", 1e-4), ("weight", 3), ("xweight", 2), ("majorana", 6),
          ("wdamped", 0.5, 1e-4), ("xwdamped", 0.5, 1e-4),
          ("comp", [("weight", 4), ("coeff", 1e-6)])]


def _o(N, terms, **kw):
    return orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()], **kw)


def test_single_rotation_parity():
    rng = random.Random(31)
    N = 8
    for th in (0.0, 0.3, math.pi / 2, math.pi, -1.234):
        for _ in range(3):
            terms = rand_terms(rng, N, 40)
            g = (rng.getrandbits(N), rng.getrandbits(N))
            v = _o(N, terms)
            v.evolve1(g[0], g[1], th)
            ref = dictpath.evolve1(N, dict(terms), g, th)
            assert maxdiff(ref, v.terms()) < 1e-13
            assert v.check()


@pytest.mark.parametrize("spec", STRATS + [("adaptive", 50, 1e-12)], ids=str)
def test_sequence_parity_window1(spec):
    N = 8
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 3, 0): 1.0}
    ref, _ = dictpath.evolve_seq(N, dict(O0), gens, angs, spec)
    v = _o(N, O0)
    if spec[0] == "adaptive":
        v.evolve(gens, angs, window=1, adaptive=(spec[1], spec[2]))
    else:
        v.evolve(gens, angs, window=1, strict=filt(spec))
    assert maxdiff(ref, v.terms()) < 1e-12
    assert v.check()


def test_correction_parity_window1():
    N = 8
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 3, 0): 1.0}
    ket = 0b1010
    spec = ("comp", [("weight", 3), ("coeff", 1e-5)])
    ref, acc_ref = dictpath.evolve_seq(N, dict(O0), gens, angs, spec, energy_ket=ket)
    v = _o(N, O0)
    acc, _ = v.evolve(gens, angs, window=1, strict=filt(spec), energy_ket=ket)
    assert abs(acc_ref) > 0
    assert acc == pytest.approx(acc_ref, abs=1e-11, rel=1e-9)
    assert maxdiff(ref, v.terms()) < 1e-12


def test_windowed_cadence():
    N = 6
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 2, 0): 1.0}
    v1 = _o(N, O0)
    v1.evolve(gens, angs, window=1)
    for w in (3, 7, len(gens)):
        vw = _o(N, O0)
        vw.evolve(gens, angs, window=w)
        assert maxdiff(v1.terms(), vw.terms()) < 1e-10
    # truncated window=w equals the Dict path truncating every w rotations
    w = 5
    spec = ("weight", 3)
    ref = dict(O0)
    for i, (g, th) in enumerate(zip(gens, angs), 1):
        dictpath.evolve1(N, ref, g, th)
        if i % w == 0 or i == len(gens):
            dictpath.truncate(ref, spec)
    vw = _o(N, O0, capacity_factor=5000, append_factor=10)
    nwin = -(-len(gens) // w)
    _, ctr = vw.evolve(gens, angs, window=w, strict=filt(spec), nwin=nwin)
    assert ctr[3].sum() == 0
    assert maxdiff(ref, vw.terms()) < 1e-12
    # local weight truncation is exact at append time
    spec = ("weight", 2)
    refv = _o(N, O0)
    refv.evolve(gens, angs, window=1, strict=filt(spec))
    vl = _o(N, O0)
    vl.evolve(gens, angs, window=1, strict=filt(spec), local=filt(spec))
    assert maxdiff(refv.terms(), vl.terms()) < 1e-11


def test_early_merge_tight_capacity():
    N = 8
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 3, 0): 1.0}
    v = _o(N, O0, append_factor=0.01, min_capacity=4)
    nwin = -(-len(gens) // 10)
    _, ctr = v.evolve(gens, angs, window=10, nwin=nwin)
    assert ctr[3].sum() > 0
    ref = _o(N, O0)
    ref.evolve(gens, angs, window=1)
    assert maxdiff(ref.terms(), v.terms()) < 1e-10


@pytest.mark.parametrize("spec", [("coeff", 0.2), ("weight", 3), ("xweight", 2), ("majorana", 5),
                                  ("wdamped", 0.5, 0.05), ("xwdamped", 0.5, 0.05)], ids=str)
def test_clip_parity(spec):
    # test_spv_equivalence.jl:138-159
    rng = random.Random(21)
    N = 6
    terms = rand_terms(rng, N, 80)
    v = _o(N, terms)
    v.compact(filt(spec))
    ref = dictpath.truncate(dict(terms), spec)
    assert v.terms() == ref
    assert v.check()


def test_channels_parity_subsets():
    # test_spv_equivalence.jl:196-218 (qubits=[1,3] subsets)
    rng = random.Random(4)
    N = 6
    terms = rand_terms(rng, N, 40)
    for kind, prm in ((4, [0.01, 0.02, 0.03]), (0, [0.05]), (1, [0.05]), (2, [0.05]), (3, [0.05])):
        for mask in (None, 0b101):
            v = _o(N, terms)
            v.channel(kind, prm, mask)
            got = v.terms()
            M = mask if mask is not None else (1 << N) - 1
            for (z, x), c in terms.items():
                if kind == 4:
                    pX, pY, pZ = prm
                    lX, lY, lZ = 1 - 2 * (pY + pZ), 1 - 2 * (pX + pZ), 1 - 2 * (pX + pY)
                    nX = bin(x & M & ~z).count("1"); nY = bin(x & M & z).count("1"); nZ = bin(z & M & ~x).count("1")
                    f = lX**nX * lY**nY * lZ**nZ
                else:
                    p = prm[0]
                    lam = 1 - 4 * p / 3 if kind == 0 else 1 - 2 * p
                    sel = [(z | x), x, z, x ^ z][kind] & M
                    f = lam ** bin(sel).count("1")
                assert got[(z, x)] == pytest.approx(c * f, rel=1e-14)
