"""Independent Dict-path restatement (test helper, not product code).

PauliSum evolve!/truncate! of src/evolve.jl:226-240 and src/evolve.jl:305-315,
with the clip predicates of src/clip.jl, computed WITHOUT the packed-word tricks
of the SparsePauliVector kernels: products of Pauli strings are formed qubit by
qubit from the single-qubit multiplication table, and the Majorana weight by
the per-bit control-flag scan the reference's docstring describes
(src/clip.jl:82-86).  Used to cross-check the C oracle.
"""
import math

# single-qubit (z, x) -> label; product table a*b = phase * c with phase in {1, 1j, -1, -1j}
_LBL = {(0, 0): "I", (0, 1): "X", (1, 0): "Z", (1, 1): "Y"}
_BITS = {v: k for k, v in _LBL.items()}
_MUL = {}
for a in "IXYZ":
    for b in "IXYZ":
        if a == "I":
            _MUL[a, b] = (1, b)
        elif b == "I":
            _MUL[a, b] = (1, a)
        elif a == b:
            _MUL[a, b] = (1, "I")
for (a, b, c) in (("X", "Y", "Z"), ("Y", "Z", "X"), ("Z", "X", "Y")):
    _MUL[a, b] = (1j, c)
    _MUL[b, a] = (-1j, c)


def pauli_mul(N, g, p):
    """(phase, key) of the product G*P of two Hermitian Pauli strings."""
    ph = 1
    z = x = 0
    for q in range(N):
        a = _LBL[((g[0] >> q) & 1, (g[1] >> q) & 1)]
        b = _LBL[((p[0] >> q) & 1, (p[1] >> q) & 1)]
        f, c = _MUL[a, b]
        ph *= f
        zb, xb = _BITS[c]
        z |= zb << q
        x |= xb << q
    return ph, (z, x)


def commute(N, g, p):
    ph, _ = pauli_mul(N, g, p)
    ph2, _ = pauli_mul(N, p, g)
    return ph == ph2


def evolve1(N, O, g, theta):
    """evolve!(O::PauliSum, G, θ) (evolve.jl:226-240), real coefficients."""
    cs, sn = math.cos(theta), math.sin(theta)
    sin_branch = {}
    for p, c in list(O.items()):
        if not commute(N, g, p):
            ph, k = pauli_mul(N, g, p)
            val = c * 1j * sn * ph
            assert abs(val.imag) == 0.0
            sin_branch[k] = sin_branch.get(k, 0.0) + val.real
            O[p] = c * cs
    for k, v in sin_branch.items():
        O[k] = O.get(k, 0.0) + v
    return O


def weight(k):
    return bin(k[0] | k[1]).count("1")


def x_weight(k):
    return bin(k[1]).count("1")


def majorana_weight(k):
    z, x = k
    w = 0
    ctrl = True
    for j in range(127, -1, -1):
        xb, zb = (x >> j) & 1, (z >> j) & 1
        if xb:
            w += 1
        elif zb:
            w += 2 if ctrl else 0
        else:
            w += 0 if ctrl else 2
        if xb:
            ctrl = not ctrl
    return w


def keep(strategy, k, c):
    """Per-term keep decision of one compilable strategy (clip.jl predicates)."""
    kind = strategy[0]
    if kind == "none":
        return True
    if kind == "coeff":
        return abs(c) > strategy[1]
    if kind == "weight":
        return weight(k) <= strategy[1]
    if kind == "xweight":
        return x_weight(k) <= strategy[1]
    if kind == "majorana":
        return majorana_weight(k) <= strategy[1]
    if kind == "wdamped":
        return abs(c) * math.exp(-strategy[1] * weight(k)) > strategy[2]
    if kind == "xwdamped":
        return abs(c) * math.exp(-strategy[1] * x_weight(k)) > strategy[2]
    raise ValueError(kind)


def truncate(O, strategy):
    """truncate!(O, strategy) for simple, composite ('comp', [...]) and adaptive strategies."""
    kind = strategy[0]
    if kind == "comp":
        for s in strategy[1]:
            truncate(O, s)
        return O
    if kind == "adaptive":
        max_terms, min_thresh = strategy[1], strategy[2]
        if len(O) > max_terms:
            coeffs = sorted(abs(v) for v in O.values())
            thr = coeffs[len(coeffs) - max_terms - 1]
            for k in [k for k, v in O.items() if not abs(v) > thr]:
                del O[k]
        else:
            for k in [k for k, v in O.items() if not abs(v) > min_thresh]:
                del O[k]
        return O
    for k in [k for k, v in O.items() if not keep(strategy, k, v)]:
        del O[k]
    return O


def expectation(O, ket):
    s = 0.0
    for (z, x), c in O.items():
        if x == 0:
            s += (-1) ** bin(z & ket).count("1") * c
    return s


def evolve_seq(N, O, gens, angles, strategy=("none",), energy_ket=None):
    """evolve(O, gens, angles; truncation, correction) (evolve.jl:305-315)."""
    acc = 0.0
    for g, th in zip(gens, angles):
        evolve1(N, O, g, th)
        if energy_ket is not None:
            before = expectation(O, energy_ket)
        truncate(O, strategy)
        if energy_ket is not None:
            acc += expectation(O, energy_ket) - before
    return O, acc
