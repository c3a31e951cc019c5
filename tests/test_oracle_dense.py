"""Pins the CPU oracle to exact linear algebra: Heisenberg conjugation by dense
matrices (test_evolution.jl / test_spv_evolution.jl style, N <= 5) and the
channels by brute-force Kraus sums (test_channels.jl:185-240, N <= 3)."""
import math
import random

import numpy as np
import pytest

import orc
from helpers import CHANNEL_KIND, rand_terms

I2 = np.eye(2, dtype=complex)
X2 = np.array([[0, 1], [1, 0]], dtype=complex)
Y2 = np.array([[0, -1j], [1j, 0]], dtype=complex)
Z2 = np.array([[1, 0], [0, -1]], dtype=complex)


def pmat(N, z, x):
    """Dense matrix of the Hermitian Pauli string (z, x); qubit 1 = least significant factor."""
    m = np.ones((1, 1), dtype=complex)
    for q in range(N):
        zb, xb = (z >> q) & 1, (x >> q) & 1
        s = Y2 if (zb and xb) else X2 if xb else Z2 if zb else I2
        m = np.kron(s, m)
    return m


def to_dense(N, terms):
    return sum(c * pmat(N, z, x) for (z, x), c in terms.items()) if terms else np.zeros((2**N, 2**N), complex)


def decompose(N, M):
    out = {}
    for z in range(2**N):
        for x in range(2**N):
            c = np.trace(pmat(N, z, x) @ M) / 2**N
            if abs(c) > 1e-14:
                assert abs(c.imag) < 1e-12
                out[(z, x)] = c.real
    return out


@pytest.mark.parametrize("seed", range(6))
def test_single_rotation_dense(seed):
    rng = random.Random(seed)
    N = 4
    terms = rand_terms(rng, N, 8)
    g = (rng.getrandbits(N), rng.getrandbits(N))
    if g == (0, 0):
        g = (1, 0)
    th = rng.uniform(-math.pi, math.pi)
    v = orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()])
    v.evolve1(g[0], g[1], th)
    G = pmat(N, *g)
    U = math.cos(th / 2) * np.eye(2**N) - 1j * math.sin(th / 2) * G
    ref = decompose(N, U.conj().T @ to_dense(N, terms) @ U)
    got = v.terms()
    for k in set(ref) | set(got):
        assert abs(ref.get(k, 0.0) - got.get(k, 0.0)) < 1e-12


def test_sequence_dense():
    rng = random.Random(7)
    N = 3
    terms = rand_terms(rng, N, 5)
    gens = [(rng.getrandbits(N), rng.getrandbits(N)) for _ in range(12)]
    angs = [rng.uniform(-1, 1) for _ in gens]
    v = orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()])
    v.evolve(gens, angs, window=1)
    M = to_dense(N, terms)
    for g, th in zip(gens, angs):
        U = math.cos(th / 2) * np.eye(2**N) - 1j * math.sin(th / 2) * pmat(N, *g)
        M = U.conj().T @ M @ U
    ref = decompose(N, M)
    got = v.terms()
    for k in set(ref) | set(got):
        assert abs(ref.get(k, 0.0) - got.get(k, 0.0)) < 1e-12


def kraus(N, pI, pX, pY, pZ, qubits):
    ks = []
    qs = sorted(qubits)
    for idx in range(4 ** len(qs)):
        coef = 1.0
        m = np.ones((1, 1), dtype=complex)
        a = 0
        for q in range(1, N + 1):
            if q in qs:
                ch = (idx // 4**a) % 4
                coef *= math.sqrt((pI, pX, pY, pZ)[ch])
                m = np.kron((I2, X2, Y2, Z2)[ch], m)
                a += 1
            else:
                m = np.kron(I2, m)
        ks.append(coef * m)
    return ks


WEIGHTS = {
    "depolarizing": lambda p: (1 - p, p / 3, p / 3, p / 3),
    "dephasing": lambda p: (1 - p, 0.0, 0.0, p),
    "bit_flip": lambda p: (1 - p, p, 0.0, 0.0),
    "bit_phase_flip": lambda p: (1 - p, 0.0, p, 0.0),
}


@pytest.mark.parametrize("N", [1, 2, 3])
@pytest.mark.parametrize("name", list(WEIGHTS))
def test_channel_kraus(N, name):
    rng = random.Random(N * 31 + len(name))
    for p in (0.0, 0.07, 0.3, 0.55, 0.91, 1.0):
        terms = rand_terms(rng, N, min(2**N, 4**N))
        v = orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()])
        v.channel(CHANNEL_KIND[name], [p])
        ks = kraus(N, *WEIGHTS[name](p), qubits=range(1, N + 1))
        M = to_dense(N, terms)
        ref = sum(K.conj().T @ M @ K for K in ks)
        assert np.linalg.norm(to_dense(N, v.terms()) - ref) < 1e-11


@pytest.mark.parametrize("N", [2, 3])
def test_pauli_channel_subsets_kraus(N):
    rng = random.Random(N)
    for qubits in ([1], [N], list(range(1, N + 1)), [1, N]):
        for (pX, pY, pZ) in ((0.0, 0.0, 0.0), (0.1, 0.2, 0.3), (0.4, 0.0, 0.4)):
            terms = rand_terms(rng, N, 2**N)
            v = orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()])
            mask = sum(1 << (q - 1) for q in qubits)
            v.channel(4, [pX, pY, pZ], mask)
            ks = kraus(N, 1 - pX - pY - pZ, pX, pY, pZ, qubits)
            M = to_dense(N, terms)
            ref = sum(K.conj().T @ M @ K for K in ks)
            assert np.linalg.norm(to_dense(N, v.terms()) - ref) < 1e-11


def test_jl_pow_accuracy():
    # the compensated power is within one ulp of the exactly rounded value
    from fractions import Fraction
    for lam in (1 - 4 * 0.1 / 3, 0.999, 1 - 2 * 5e-4, 0.37, 1.7):
        for k in range(0, 40):
            exact = Fraction(lam) ** k
            got = orc.jl_pow(lam, k)
            assert abs(Fraction(got) - exact) <= Fraction(math.ulp(float(exact)))
