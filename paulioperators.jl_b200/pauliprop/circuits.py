"""Seeded synthetic workloads (Trotterised Ising-type circuits in Heisenberg order).

Conventions: qubit q is 1-based and maps to bit q-1; RZZ(θ) on (i, j) is the
rotation exp(iθ/2 Z_i Z_j) applied as evolve!(v, Z_i Z_j, θ); RX(θ) on q is
evolve!(v, X_q, θ).  Each layer lists its generators in the order written
(RZZ edges, then RX sites) and is repeated `layers` times.  All randomness comes
from a splitmix64 stream so that every consumer (GPU engine, CPU oracle, bench)
sees the same instance for the same seed.
"""
import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

from .paulis import PauliBasis

M64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014): 64-bit state, Weyl increment + mix."""

    def __init__(self, seed):
        self.s = int(seed) & M64

    def next_u64(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def uniform(self, lo=0.0, hi=1.0):
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / 9007199254740992.0))

    def randint(self, n):
        """Uniform integer in [0, n)."""
        return self.next_u64() % n

    def shuffle(self, a):
        for i in range(len(a) - 1, 0, -1):
            j = self.randint(i + 1)
            a[i], a[j] = a[j], a[i]
        return a


@dataclass
class Workload:
    name: str
    N: int
    layer: List[PauliBasis]
    angles: List[float]
    layers: int
    observable: List[Tuple[int, int, float]]      # (z, x, coefficient)
    thresh: float
    wmax: Optional[int]
    channel: Optional[Tuple[str, float]] = None   # applied after every layer
    seed: int = 0
    meta: dict = field(default_factory=dict)

    def generators(self):
        return self.layer * self.layers, self.angles * self.layers

    @property
    def rotations(self):
        return len(self.layer) * self.layers


def zz(N, i, j):
    return PauliBasis(N, (1 << (i - 1)) | (1 << (j - 1)), 0)


def xq(N, q):
    return PauliBasis(N, 0, 1 << (q - 1))


def chain20(layers=8, theta_j=0.3, theta_h=0.2, thresh=1e-5):
    """N=20 open chain, observable Z_10: 19 RZZ(θ_J) on (i,i+1), then RX(θ_h) on all."""
    N = 20
    layer, ang = [], []
    for i in range(1, N):
        layer.append(zz(N, i, i + 1)); ang.append(theta_j)
    for q in range(1, N + 1):
        layer.append(xq(N, q)); ang.append(theta_h)
    return Workload("chain20", N, layer, ang, layers, [(1 << 9, 0, 1.0)], thresh, None)


def lattice_edges(R=8, Cn=8):
    """8x8 open lattice, q = 8r + c + 1: horizontal edges row by row, then vertical."""
    q = lambda r, c: Cn * r + c + 1
    edges = [(q(r, c), q(r, c + 1)) for r in range(R) for c in range(Cn - 1)]
    edges += [(q(r, c), q(r + 1, c)) for r in range(R - 1) for c in range(Cn)]
    return edges


def lattice64(layers=20, theta_j=0.3, theta_h=0.25, thresh=1e-5, wmax=12, p_depol=1e-3):
    """N=64 8x8 lattice, observable mean Z (64 terms, 1/64), depolarizing after each layer."""
    N = 64
    layer, ang = [], []
    for (i, j) in lattice_edges():
        layer.append(zz(N, i, j)); ang.append(theta_j)
    for qq in range(1, N + 1):
        layer.append(xq(N, qq)); ang.append(theta_h)
    obs = [(1 << (qq - 1), 0, 1.0 / 64) for qq in range(1, N + 1)]
    return Workload("lattice64", N, layer, ang, layers, obs, thresh, wmax,
                    channel=("depolarizing", p_depol) if p_depol else None)


def _graph_edges(N, seed, n_edges):
    rng = SplitMix64(seed)
    cand = [(i, j) for i in range(1, N + 1) for j in range(i + 1, N + 1)]
    rng.shuffle(cand)
    deg = [0] * (N + 1)
    edges = []
    for (i, j) in cand:
        if deg[i] < 3 and deg[j] < 3:
            edges.append((i, j)); deg[i] += 1; deg[j] += 1
            if len(edges) == n_edges:
                break
    return edges


def default_graph_seed(N=127, n_edges=144, obs_qubit=63, start=127):
    """First seed >= 127 whose graph gives the observable's qubit degree 3.  With 144
    edges on 127 qubits about a tenth of the qubits stay isolated, and an isolated
    observable qubit would make the workload trivial (2 terms)."""
    s = start
    while sum(1 for e in _graph_edges(N, s, n_edges) if obs_qubit in e) != 3:
        s += 1
    return s


def random_graph127(seed=None, layers=24, thresh=1e-4, wmax=10, p_deph=5e-4, n_edges=144):
    """N=127 random graph, max degree 3, exactly 144 edges; θ_J~U[0.1,0.5] per edge,
    θ_h~U[0,π/4] per qubit (drawn once); observable Z_63; dephasing after each layer."""
    N = 127
    if seed is None:
        seed = default_graph_seed(N, n_edges)
    rng = SplitMix64(seed)
    cand = [(i, j) for i in range(1, N + 1) for j in range(i + 1, N + 1)]
    rng.shuffle(cand)
    deg = [0] * (N + 1)
    edges = []
    for (i, j) in cand:
        if deg[i] < 3 and deg[j] < 3:
            edges.append((i, j)); deg[i] += 1; deg[j] += 1
            if len(edges) == n_edges:
                break
    th_j = [rng.uniform(0.1, 0.5) for _ in edges]
    th_h = [rng.uniform(0.0, math.pi / 4) for _ in range(N)]
    layer = [zz(N, i, j) for (i, j) in edges] + [xq(N, q) for q in range(1, N + 1)]
    ang = th_j + th_h
    return Workload("graph127", N, layer, ang, layers, [(1 << 62, 0, 1.0)], thresh, wmax,
                    channel=("dephasing", p_deph) if p_deph else None, seed=seed,
                    meta={"edges": edges})


def batch_instances(count=256, seed=5, thresh=1e-5):
    """Uneven instances on the 8x8 lattice: depth U{4..24}, θ_J, θ_h ~ U[0.05, 0.5],
    observable a random Pauli string of weight 1-4 (seeded sites and types)."""
    rng = SplitMix64(seed)
    N = 64
    out = []
    edges = lattice_edges()
    for k in range(count):
        depth = 4 + rng.randint(21)
        tj = rng.uniform(0.05, 0.5)
        th = rng.uniform(0.05, 0.5)
        w = 1 + rng.randint(4)
        sites = rng.shuffle(list(range(1, N + 1)))[:w]
        z = x = 0
        for s in sites:
            t = rng.randint(3)
            if t in (0, 1):
                x |= 1 << (s - 1)
            if t in (1, 2):
                z |= 1 << (s - 1)
        layer = [zz(N, i, j) for (i, j) in edges] + [xq(N, q) for q in range(1, N + 1)]
        ang = [tj] * len(edges) + [th] * N
        out.append(Workload(f"inst{k}", N, layer, ang, depth, [(z, x, 1.0)], thresh, None, seed=seed))
    return out


def heisenberg_chain_terms(N, Jx=1.0, Jy=0.7, Jz=1.1, hz=0.3):
    """Terms of the reference tests' Heisenberg chain (test_spv_evolution.jl:16-27)."""
    terms = []
    for i in range(1, N):
        terms.append((PauliBasis.from_sites(N, X=[i, i + 1]), Jx))
        terms.append((PauliBasis.from_sites(N, Y=[i, i + 1]), Jy))
        terms.append((PauliBasis.from_sites(N, Z=[i, i + 1]), Jz))
    for i in range(1, N + 1):
        terms.append((PauliBasis.from_sites(N, Z=[i]), hz))
    return terms


def trotterize(terms, dt, n_trotter=1, order=1):
    """trotterize (decompose.jl:22-53) over an ordered list of (PauliBasis, c)."""
    if order not in (1, 2):
        raise ValueError("Only order=1 and order=2 Trotter decompositions are supported")
    gens, angles = [], []
    step = dt / n_trotter
    for _ in range(n_trotter):
        if order == 1:
            for P, c in terms:
                gens.append(P); angles.append(2 * step * c)
        else:
            for P, c in terms:
                gens.append(P); angles.append(step * c)
            for P, c in reversed(terms):
                gens.append(P); angles.append(step * c)
    return gens, angles
