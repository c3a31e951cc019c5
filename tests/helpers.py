"""Shared test helpers: strategy specs, seeded instances, comparisons."""
import math
import random

import numpy as np

import pauliprop as pp

INT64_MAX = 2**63 - 1


def strategy(spec):
    """JSON/tuple spec -> pauliprop strategy object."""
    k = spec[0]
    if k == "none":
        return pp.NoTruncation()
    if k == "coeff":
        return pp.CoeffTruncation(spec[1])
    if k == "weight":
        return pp.WeightTruncation(spec[1])
    if k == "xweight":
        return pp.XWeightTruncation(spec[1])
    if k == "majorana":
        return pp.MajoranaWeightTruncation(spec[1])
    if k == "wdamped":
        return pp.WeightDampedTruncation(spec[1], spec[2])
    if k == "xwdamped":
        return pp.XWeightDampedTruncation(spec[1], spec[2])
    if k == "comp":
        return pp.CompositeTruncation(*[strategy(s) for s in spec[1]])
    if k == "adaptive":
        return pp.AdaptiveTruncation(spec[1], spec[2])
    raise ValueError(k)


def filt(spec):
    return tuple(pp.compile_filter(strategy(spec)))


def key_of(s):
    b = pp.PauliBasis.from_string(s)
    return (b.z, b.x)


def rand_terms(rng, N, n, real=True, scale=1.0):
    n = min(n, 4**N // 2)   # never ask for more distinct keys than the space holds
    out = {}
    while len(out) < n:
        out[(rng.getrandbits(N), rng.getrandbits(N))] = scale * (rng.random() - 0.5)
    return out


def maxdiff(a, b):
    """_maxdiff (test_spv_evolution.jl:8-14): max |difference| over the key union."""
    keys = set(a) | set(b)
    if not keys:
        return 0.0
    return max(abs(a.get(k, 0.0) - b.get(k, 0.0)) for k in keys)


def heisenberg_gens(N, dt=0.05, n_trotter=2, order=2):
    terms = pp.circuits.heisenberg_chain_terms(N)
    g, a = pp.circuits.trotterize(terms, dt, n_trotter=n_trotter, order=order)
    return [(p.z, p.x) for p in g], a


def mask_bits(N, qubits):
    return pp.qubit_mask(N, qubits)


CHANNEL_KIND = {"depolarizing": 0, "dephasing": 1, "bit_flip": 2, "bit_phase_flip": 3, "pauli": 4}
