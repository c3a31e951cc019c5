"""SparsePauliVector algebra (spv_ops.jl) on the GPU for real (Float64)
coefficients, against restatements of the reference functions: scalar multiply,
norm, tr, sum! / + / -, inner_product, products and anticommutators, and the
errors the reference raises for a real-typed vector (commutator, imaginary
products).  Keys bit-exact; a sum of two coefficients (sum!, +, -) bit-exact;
longer sums (products) within 1e-12 relative."""
import math
import random

import numpy as np
import pytest

import pauliprop as pp
from helpers import rand_terms

pytestmark = pytest.mark.gpu


def vec(N, terms):
    z, x = pp.pack_keys(N, list(terms))
    c = np.array(list(terms.values()), dtype=np.float64)
    v = pp.SparsePauliVector(N, max(16, 2 * len(c)), max(16, 2 * len(c)))
    v.upload(z, x, c, sorted=False)
    return v


def terms_of(v):
    return {k: c for k, c in v.to_paulisum().items()}


def phase_k(az, ax, bz, bx):
    zp, xp = az ^ bz, ax ^ bx
    pc = lambda t: bin(t).count("1")
    return (pc(zp & xp) - pc(az & ax) - pc(bz & bx) + 2 * pc(ax & bz)) % 4


def product_ref(A, B, kind):
    """_mul_spv / _commutator_triples!(anti) + _triples_to_live! for real T."""
    out = {}
    for (az, ax), ca in sorted(A.items()):
        for (bz, bx), cb in sorted(B.items()):
            k = phase_k(az, ax, bz, bx)
            if kind == 0:
                assert k % 2 == 0
                c = (ca if k == 0 else -ca) * cb
            else:
                if k % 2:
                    continue
                c = (2 * (1 - k) * ca) * cb
            key = (az ^ bz, ax ^ bx)
            out[key] = out.get(key, 0.0) + c
    return out


def close(got, ref, scale):
    assert set(got) == set(ref)
    for k in ref:
        assert abs(got[k] - ref[k]) <= 1e-12 * scale, (k, got[k], ref[k])


@pytest.mark.parametrize("N", [8, 70])
def test_scalar_norm_trace(N):
    rng = random.Random(N)
    terms = rand_terms(rng, N, 500)
    terms[(0, 0)] = 0.75
    v = vec(N, terms)
    c = np.array(list(terms.values()))
    assert abs(pp.norm(v) - math.sqrt(float(np.sum(c * c)))) <= 1e-12 * math.sqrt(float(np.sum(c * c)))
    assert abs(pp.norm(v, 1) - float(np.sum(np.abs(c)))) <= 1e-12 * float(np.sum(np.abs(c)))
    assert pp.norm(v, math.inf) == float(np.max(np.abs(c)))
    assert abs(pp.norm(v, 3) - float(np.sum(np.abs(c) ** 3)) ** (1 / 3)) <= 1e-12
    # tr: identity coefficient times the reference's Int64 2^N (wraps to 0 for N >= 64)
    assert pp.tr(v) == (0.75 * 2.0 ** N if N < 63 else 0.0)
    w = pp.scaled(v, -2.5)
    gz, gx, gc = w.to_arrays()
    oz, ox, oc = v.to_arrays()
    assert np.array_equal(gz, oz) and np.array_equal(gc, oc * -2.5)
    assert np.array_equal((-v).to_arrays()[2], -oc)


@pytest.mark.parametrize("N", [10, 64, 100])
def test_sum_add_sub(N):
    rng = random.Random(N + 1)
    A = rand_terms(rng, N, 3000)
    B = rand_terms(rng, N, 2000)
    for k in list(A)[:300]:
        B[k] = -A[k] if rng.random() < 0.5 else rng.random()   # shared keys, some cancelling to 0
    a, b = vec(N, A), vec(N, B)
    for op, sign in ((pp.add, 1.0), (pp.sub, -1.0)):
        got = terms_of(op(a, b))
        ref = dict(A)
        for k, c in B.items():
            ref[k] = ref[k] + sign * c if k in ref else sign * c
        assert set(got) == set(ref)
        assert all(got[k] == ref[k] for k in ref)          # one IEEE add each: bit-exact
    s = a.copy()
    pp.sum_(s, b)
    assert terms_of(s) == terms_of(a + b)
    pp.check_spv(s)
    assert sum(1 for c in terms_of(a + b).values() if c == 0.0) > 0   # zeros kept (Dict parity)


@pytest.mark.parametrize("N", [12, 90])
def test_inner_product(N):
    rng = random.Random(N + 2)
    A = rand_terms(rng, N, 4000)
    B = rand_terms(rng, N, 3000)
    for k in list(A)[:1000]:
        B[k] = rng.random() - 0.5
    ref = sum(A[k] * B[k] for k in sorted(A) if k in B)
    got = pp.inner_product(vec(N, A), vec(N, B))
    assert abs(got - ref) <= 1e-12 * sum(abs(A[k] * B[k]) for k in A if k in B)


@pytest.mark.parametrize("N", [8, 66])
def test_product_of_diagonal_operators(N):
    rng = random.Random(N + 3)
    A = {(rng.getrandbits(N), 0): rng.random() - 0.5 for _ in range(60)}
    B = {(rng.getrandbits(N), 0): rng.random() - 0.5 for _ in range(50)}
    got = terms_of(vec(N, A) * vec(N, B))
    close(got, product_ref(A, B, 0), max(1.0, sum(abs(c) for c in A.values()) * sum(abs(c) for c in B.values())))


def test_product_with_imaginary_coefficients_raises():
    A = {(1, 0): 1.0}          # Z1
    B = {(0, 1): 1.0}          # X1: ZX = iY
    with pytest.raises(pp.PauliPropError):
        vec(3, A) * vec(3, B)
    with pytest.raises(pp.PauliPropError):
        pp.commutator(vec(3, A), vec(3, B))


@pytest.mark.parametrize("N", [6, 70])
def test_anticommutator(N):
    rng = random.Random(N + 4)
    A = rand_terms(rng, N, 120)
    B = rand_terms(rng, N, 90)
    got = terms_of(pp.anticommutator(vec(N, A), vec(N, B)))
    ref = product_ref(A, B, 1)
    close(got, ref, max(1.0, 2 * sum(abs(c) for c in A.values()) * sum(abs(c) for c in B.values())))
    # {P, P} = 2 I for a single Pauli with coefficient 1
    p = {(5, 3): 1.0}
    assert terms_of(pp.anticommutator(vec(N, p), vec(N, p))) == {(0, 0): 2.0}
