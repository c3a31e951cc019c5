"""GPU parity: libpauliprop (through its C ABI) against the CPU oracle on the same
seeded inputs.  Bar: bit-exact surviving key sets; coefficients within
1e-12 * max(1, max|c|) (they are in fact bit-identical at window = 1, asserted
where the arithmetic is identical); expectation values within
1e-12 * sum_{x=0}|c| (the condition-number-aware relative bound for a sum)."""
import json
import math
import os
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import CHANNEL_KIND, filt, heisenberg_gens, key_of, maxdiff, rand_terms, strategy

pytestmark = pytest.mark.gpu

COEF_TOL = 1e-12
STRATS = [("none",), ("coeff", 1e-4), ("weight", 3), ("xweight", 2), ("majorana", 6),
          ("wdamped", 0.5, 1e-4), ("xwdamped", 0.5, 1e-4),
          ("comp", [("weight", 4), ("coeff", 1e-6)])]


def gpu_from_oracle(v, N, live_cap=None, append_cap=None, sorted=True):
    z, x, c = v.arrays()
    g = pp.SparsePauliVector(N, live_cap or max(16, 2 * len(c)), append_cap or max(16, 2 * len(c)))
    g.upload(z, x, c, sorted=sorted)
    return g


def compare(g, v, bitexact=False, tol=COEF_TOL):
    gz, gx, gc = g.to_arrays()
    oz, ox, oc = v.arrays()
    assert gz.shape == oz.shape, (gz.shape, oz.shape)
    assert np.array_equal(gz, oz) and np.array_equal(gx, ox), "surviving key sets differ"
    scale = max(1.0, float(np.abs(oc).max()) if len(oc) else 1.0)
    assert np.abs(gc - oc).max(initial=0.0) <= tol * scale
    if bitexact:
        assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64)), "coefficients not bit-identical"
    pp.check_spv(g)


def oracle_from_terms(N, terms, **kw):
    return orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()], **kw)


def expect_bound(v, ket=0):
    z, x, c = v.arrays()
    diag = np.all(x == 0, axis=1)
    return 1e-12 * max(1e-300, float(np.abs(c[diag]).sum()))


# ------------------------------------------------------------------ basics
@pytest.mark.parametrize("N", [8, 64, 70, 128])
def test_upload_sort_download(N):
    rng = random.Random(N)
    terms = rand_terms(rng, N, 3000)
    keys = list(terms)
    rng.shuffle(keys)
    z, x = pp.pack_keys(N, keys)
    c = np.array([terms[k] for k in keys])
    g = pp.SparsePauliVector(N, 16, 16)
    g.upload(z, x, c, sorted=False)
    v = oracle_from_terms(N, terms)
    compare(g, v, bitexact=True)
    assert len(g) == 3000


def test_empty_and_single():
    g = pp.SparsePauliVector(8)
    g.upload(np.zeros(0, np.uint64), np.zeros(0, np.uint64), np.zeros(0), sorted=True)
    assert len(g) == 0
    pp.evolve_(g, pp.PauliBasis.from_string("XXIIIIII"), 0.3)
    assert len(g) == 0
    assert pp.expectation_value(g, 0) == 0.0
    g.upload(*pp.pack_keys(8, [(1, 0)]), np.array([1.0]), sorted=True)
    pp.evolve_(g, pp.PauliBasis.from_string("XIIIIIII"), 0.3)
    assert len(g) == 2
    pp.check_spv(g)


# ------------------------------------------------------------------ rotation
@pytest.mark.parametrize("N", [8, 70])
def test_single_rotation_parity(N):
    rng = random.Random(31 + N)
    for th in (0.0, 0.3, math.pi / 2, math.pi, -1.234):
        for _ in range(3):
            terms = rand_terms(rng, N, 40)
            gz_, gx_ = rng.getrandbits(N), rng.getrandbits(N)
            v = oracle_from_terms(N, terms)
            g = gpu_from_oracle(v, N)
            v.evolve1(gz_, gx_, th)
            pp.evolve_(g, pp.PauliBasis(N, gz_, gx_), th)
            compare(g, v, bitexact=True)


@pytest.mark.parametrize("N", [12, 64, 100])
def test_random_rotations_large(N):
    """Many random low-weight rotations on ~2e5 terms, exercising multi-tile scans."""
    rng = random.Random(N)
    terms = rand_terms(rng, N, 200_000)
    v = oracle_from_terms(N, terms)
    g = gpu_from_oracle(v, N)
    gens, angs = [], []
    for _ in range(12):
        q = rng.sample(range(N), 2)
        kind = rng.randrange(5)
        if kind == 0:
            gens.append(((1 << q[0]) | (1 << q[1]), 0))
        elif kind == 1:
            gens.append((0, 1 << q[0]))
        elif kind == 2:
            gens.append((1 << q[0], 1 << q[0]))
        elif kind == 3:
            gens.append(((1 << q[0]) | (1 << q[1]), (1 << q[0]) | (1 << q[1])))
        else:
            gens.append((rng.getrandbits(N), rng.getrandbits(N)))
        angs.append(rng.uniform(-2, 2))
    f = filt(("coeff", 1e-7))
    v.evolve(gens, angs, window=1, strict=f)
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(("coeff", 1e-7)))
    compare(g, v, bitexact=True)


@pytest.mark.parametrize("spec", STRATS, ids=str)
@pytest.mark.parametrize("shift", [0, 60])
def test_sequence_parity_window1(spec, shift):
    N = 8 + shift
    gens, angs = heisenberg_gens(8)
    gens = [(z << shift, x << shift) for z, x in gens]
    O0 = {(1 << (3 + shift), 0): 1.0}
    v = oracle_from_terms(N, O0)
    g = gpu_from_oracle(v, N, append_cap=v.append_cap)
    v.evolve(gens, angs, window=1, strict=filt(spec))
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(spec))
    compare(g, v, bitexact=True)


def test_correction_parity_window1():
    N = 8
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 3, 0): 1.0}
    spec = ("comp", [("weight", 3), ("coeff", 1e-5)])
    v = oracle_from_terms(N, O0)
    g = gpu_from_oracle(v, N, append_cap=v.append_cap)
    acc_o, _ = v.evolve(gens, angs, window=1, strict=filt(spec), energy_ket=0b1010)
    corr = pp.EnergyCorrection(0b1010)
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(spec), correction=corr)
    assert abs(acc_o) > 0
    assert corr.accumulated_energy == pytest.approx(acc_o, abs=1e-11, rel=1e-9)
    compare(g, v, bitexact=True)


def test_window1_early_merge_prefilter():
    """n > append capacity at window 1 triggers the reference's early boundary, which
    applies the strict filter to live terms before the rotation (spv_evolve.jl:356-362)."""
    rng = random.Random(5)
    N = 10
    terms = rand_terms(rng, N, 300)
    for k in list(terms)[:100]:
        terms[k] = 1e-9 * (rng.random() - 0.5)       # below the threshold before any rotation
    gens = [((1 << 1) | (1 << 2), 0), (0, 1 << 4), ((1 << 3) | (1 << 7), 0)] * 4
    angs = [0.4, 0.3, -0.7] * 4
    spec = ("coeff", 1e-6)
    v = oracle_from_terms(N, terms, append_factor=0.1, min_capacity=4)
    g = gpu_from_oracle(v, N, append_cap=v.append_cap)
    acc_o, ctr = v.evolve(gens, angs, window=1, strict=filt(spec), energy_ket=0, nwin=len(gens))
    assert ctr[3].sum() > 0
    corr = pp.EnergyCorrection(0)
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(spec), correction=corr)
    compare(g, v, bitexact=True)
    assert corr.accumulated_energy == pytest.approx(acc_o, abs=1e-13, rel=1e-10)


# ------------------------------------------------------------------ general path
def test_windowed_cadence_general_path():
    N = 6
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 2, 0): 1.0}
    for w in (3, 7, len(gens)):
        v = oracle_from_terms(N, O0)
        g = gpu_from_oracle(v, N, append_cap=v.append_cap)
        v.evolve(gens, angs, window=w)
        pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, window=w)
        compare(g, v, tol=1e-12)
    spec = ("weight", 3)
    v = oracle_from_terms(N, O0, capacity_factor=5000, append_factor=10)
    g = gpu_from_oracle(v, N, append_cap=v.append_cap)
    v.evolve(gens, angs, window=5, strict=filt(spec))
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, window=5, truncation=strategy(spec))
    compare(g, v)


def test_early_merge_tight_capacity_general():
    N = 8
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 3, 0): 1.0}
    v = oracle_from_terms(N, O0, append_factor=0.01, min_capacity=4)
    g = gpu_from_oracle(v, N, append_cap=v.append_cap)
    nwin = -(-len(gens) // 10)
    _, ctr = v.evolve(gens, angs, window=10, nwin=nwin)
    wc = pp.WindowCounters(nwin)
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, window=10, counters=wc)
    assert ctr[3].sum() > 0
    assert np.array_equal(wc.early_merges, ctr[3])
    assert np.array_equal(wc.merge_out, ctr[2])
    compare(g, v)


def test_local_truncation_window1():
    N = 6
    gens, angs = heisenberg_gens(N)
    O0 = {(1 << 2, 0): 1.0}
    spec = ("weight", 2)
    v = oracle_from_terms(N, O0)
    g = gpu_from_oracle(v, N, append_cap=v.append_cap)
    v.evolve(gens, angs, window=1, strict=filt(spec), local=filt(("coeff", 1e-3)))
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(spec),
               local_truncation=strategy(("coeff", 1e-3)))
    compare(g, v, bitexact=True)


def test_local_truncation_must_be_compilable():
    g = pp.SparsePauliVector(6)
    with pytest.raises(pp.ArgumentError):
        pp.evolve_(g, [pp.PauliBasis(6, 1, 0)], [0.1], local_truncation=pp.AdaptiveTruncation(10, 1e-12))
    with pytest.raises(pp.DimensionMismatch):
        pp.evolve_(g, [pp.PauliBasis(6, 1, 0)], [0.1, 0.2])
    with pytest.raises(pp.ArgumentError):
        pp.evolve_(g, [pp.PauliBasis(6, 1, 0)], [0.1], window=0)


# ------------------------------------------------------------------ clips, channels, expectation
@pytest.mark.parametrize("spec", [("coeff", 0.2), ("weight", 3), ("xweight", 2), ("majorana", 5),
                                  ("wdamped", 0.5, 0.05), ("xwdamped", 0.5, 0.05)], ids=str)
@pytest.mark.parametrize("N,n", [(6, 80), (64, 100_000), (110, 50_000)])
def test_clip_parity(spec, N, n):
    rng = random.Random(21 + N)
    terms = rand_terms(rng, N, n)
    v = oracle_from_terms(N, terms)
    g = gpu_from_oracle(v, N)
    v.compact(filt(spec))
    pp.truncate_(g, strategy(spec))
    compare(g, v, bitexact=True)


@pytest.mark.parametrize("N", [6, 64, 90])
def test_channels_parity(N):
    rng = random.Random(4 + N)
    terms = rand_terms(rng, N, 5000)
    for kind, prm in ((4, [0.01, 0.02, 0.03]), (0, [0.05]), (1, [0.05]), (2, [0.05]), (3, [0.05])):
        for qubits in (None, [1, 3]):
            v = oracle_from_terms(N, terms)
            g = gpu_from_oracle(v, N)
            mask = pp.qubit_mask(N, qubits)
            v.channel(kind, prm, mask)
            if kind == 4:
                pp.pauli_channel_(g, *prm, qubits=qubits)
            else:
                [pp.depolarizing_channel_, pp.dephasing_channel_, pp.bit_flip_channel_,
                 pp.bit_phase_flip_channel_][kind](g, prm[0], qubits=qubits)
            compare(g, v, bitexact=True)


def test_channel_argument_errors():
    g = pp.SparsePauliVector(3)
    g.upload(*pp.pack_keys(3, [key_of("XIZ")]), np.array([1.0]), sorted=True)
    for f, a in ((pp.depolarizing_channel_, (-0.1,)), (pp.depolarizing_channel_, (1.1,)),
                 (pp.dephasing_channel_, (-0.1,)), (pp.bit_flip_channel_, (2.0,)),
                 (pp.bit_phase_flip_channel_, (-1.0,)), (pp.pauli_channel_, (-0.1, 0.1, 0.1)),
                 (pp.pauli_channel_, (0.5, 0.5, 0.5))):
        with pytest.raises(pp.ArgumentError):
            f(g, *a)
    for q in ([0], [4]):
        with pytest.raises(pp.ArgumentError):
            pp.depolarizing_channel_(g, 0.1, qubits=q)


@pytest.mark.parametrize("N", [20, 64, 127])
def test_expectation(N):
    rng = random.Random(N)
    terms = rand_terms(rng, N, 50_000)
    for i, k in enumerate(list(terms)[:20_000]):
        terms[(k[0], 0)] = terms.pop(k)           # plenty of diagonal terms
    v = oracle_from_terms(N, terms)
    g = gpu_from_oracle(v, N)
    for ket in (0, rng.getrandbits(N)):
        assert abs(pp.expectation_value(g, ket) - v.expect_neumaier(ket)) <= expect_bound(v, ket)
        assert abs(pp.expectation_value(g, ket) - v.expect(ket)) <= expect_bound(v, ket)


# ------------------------------------------------------------------ golden known answers on the GPU
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))["cases"]


@pytest.mark.parametrize("case", [c for c in GOLD if c["kind"] in ("truncate", "channel")], ids=lambda c: c["name"])
def test_known_answers_gpu(case):
    N = case["N"]
    keys = [key_of(s) for s, _ in case["terms"]]
    g = pp.SparsePauliVector(N)
    g.upload(*pp.pack_keys(N, keys), np.array([c for _, c in case["terms"]]), sorted=False)
    if case["kind"] == "truncate":
        corr = pp.EnergyCorrection(0)
        pp.truncate_(g, strategy(case["strategy"]), corr)
        got = g.to_paulisum()
        assert set(got) == {key_of(s) for s in case["keep"]}
        if "energy_delta" in case:
            assert corr.accumulated_energy == pytest.approx(case["energy_delta"], abs=1e-15)
    else:
        prm = case["prm"]
        if case["channel"] == "pauli":
            pp.pauli_channel_(g, *prm)
        else:
            getattr(pp, case["channel"] + "_channel_")(g, prm[0])
        got = g.to_paulisum()
        for s, val in case["expect"].items():
            assert got[key_of(s)] == pytest.approx(val, rel=1e-14)


# ------------------------------------------------------------------ workloads
def run_workload(w, layers, fused=True):
    """Evolve a workload for `layers` layers on GPU and oracle (channel after each layer)."""
    f = filt(("comp", [("coeff", w.thresh)] + ([("weight", w.wmax)] if w.wmax else [])))
    strat = strategy(("comp", [("coeff", w.thresh)] + ([("weight", w.wmax)] if w.wmax else [])))
    v = orc.OracleSPV.from_terms(w.N, w.observable)
    g = gpu_from_oracle(v, w.N, append_cap=v.append_cap)
    gens = [(p.z, p.x) for p in w.layer]
    for _ in range(layers):
        v.evolve(gens, w.angles, window=1, strict=f)
        if w.channel:
            v.channel(CHANNEL_KIND[w.channel[0]], [w.channel[1]])
        ch = (w.channel[0], w.channel[1], None) if (w.channel and fused) else None
        pp.evolve_(g, w.layer, w.angles, truncation=strat, channel=ch)
        if w.channel and not fused:
            getattr(pp, w.channel[0] + "_channel_")(g, w.channel[1])
    return g, v


def test_config1_chain20_full():
    w = pp.circuits.chain20()
    g, v = run_workload(w, w.layers)
    compare(g, v, bitexact=True)
    assert abs(pp.expectation_value(g, 0) - v.expect(0)) <= expect_bound(v)
    assert len(g) > 100


@pytest.mark.parametrize("fused", [True, False])
def test_config2_lattice64_first_layers(fused):
    w = pp.circuits.lattice64()
    g, v = run_workload(w, 3, fused=fused)
    compare(g, v, bitexact=True)
    assert abs(pp.expectation_value(g, 0) - v.expect(0)) <= expect_bound(v)


def test_config3_graph127_first_layers():
    w = pp.circuits.random_graph127()
    g, v = run_workload(w, 2)
    compare(g, v, bitexact=True)
    assert abs(pp.expectation_value(g, 62 * 0) - v.expect(0)) <= expect_bound(v)


def test_growth_from_tiny_capacity():
    """Live buffers start tiny; the device flags each overflow and the host grows and
    resumes at the rotation that stopped, with an unchanged result."""
    w = pp.circuits.chain20()
    f = filt(("coeff", w.thresh))
    v = orc.OracleSPV.from_terms(w.N, w.observable)
    g = pp.SparsePauliVector(w.N, 1, v.append_cap)
    z, x, c = v.arrays()
    g.upload(z, x, c, sorted=True)
    gens = [(p.z, p.x) for p in w.layer]
    v.evolve(gens * 4, w.angles * 4, window=1, strict=f)
    pp.evolve_(g, w.layer * 4, w.angles * 4, truncation=strategy(("coeff", w.thresh)))
    compare(g, v, bitexact=True)


def random_rotations(rng, N, count, lo, hi):
    gens, angs = [], []
    for _ in range(count):
        i, j = rng.sample(range(N), 2)
        gens.append(((1 << i) | (1 << j), 0) if rng.random() < 0.5 else (0, 1 << i))
        angs.append(rng.uniform(lo, hi))
    return gens, angs


def test_growth_overflow_multikernel():
    """A set above the single-CTA capacity grows 3000 -> ~8e4 terms within one chunk
    of rotations from a one-term capacity: the multi-kernel path flags the overflow,
    the host grows the buffers and resumes, with an unchanged result."""
    rng = random.Random(64)
    N = 64
    terms = {}
    while len(terms) < 3000:
        terms[(rng.getrandbits(N), rng.getrandbits(N))] = rng.uniform(-1.0, 1.0)
    v = oracle_from_terms(N, terms)
    g = pp.SparsePauliVector(N, 1, v.append_cap)
    g.upload(*v.arrays(), sorted=True)
    gens, angs = random_rotations(rng, N, 8, 0.1, 1.0)
    v.evolve(gens, angs, window=1, strict=filt(("coeff", 1e-6)))
    pp.evolve_(g, [pp.PauliBasis(N, z, x) for z, x in gens], angs, truncation=strategy(("coeff", 1e-6)))
    assert len(g) > 50000
    compare(g, v, bitexact=True)


@pytest.mark.parametrize("N,n0,thresh", [(64, 3000, 0.2), (100, 1500, 0.25)])
def test_shrink_into_single_cta_path(N, n0, thresh):
    """The live set starts above the single-CTA capacity (2048 terms for N <= 64,
    1024 above) and a strong threshold shrinks it below within the first 64-rotation
    chunk: the next chunk runs in the single-CTA kernel, which reads the segment
    table the multi-kernel merge left.  Bit-exact against the oracle."""
    rng = random.Random(7)
    terms = {}
    while len(terms) < n0:
        terms[(rng.getrandbits(N), rng.getrandbits(N))] = rng.uniform(-1.0, 1.0)
    v = oracle_from_terms(N, terms)
    g = gpu_from_oracle(v, N)
    gens, angs = random_rotations(rng, N, 100, 0.05, 0.3)
    v.evolve(gens, angs, window=1, strict=filt(("coeff", thresh)))
    pp.evolve_(g, [pp.PauliBasis(N, z, x) for z, x in gens], angs, truncation=strategy(("coeff", thresh)))
    assert 0 < len(g) < (2048 if N <= 64 else 1024)
    compare(g, v, bitexact=True)


def test_copy_and_nonmutating():
    rng = random.Random(9)
    terms = rand_terms(rng, 8, 50)
    v = oracle_from_terms(8, terms)
    g = gpu_from_oracle(v, 8)
    before = g.to_paulisum()
    g2 = pp.evolve(g, pp.PauliBasis(8, 3, 5), 0.4)
    assert g.to_paulisum() == before
    v.evolve1(3, 5, 0.4)
    compare(g2, v, bitexact=True)


def test_window1_counters_match_oracle():
    """WindowCounters at window 1 (one window per rotation), including the early
    boundaries forced by the append capacity (spv_evolve.jl:356-383)."""
    rng = random.Random(11)
    N = 10
    terms = rand_terms(rng, N, 300)
    for k in list(terms)[:60]:
        terms[k] = 1e-9
    gens = [((1 << 1) | (1 << 2), 0), (0, 1 << 4), ((1 << 3) | (1 << 7), 0), (1 << 5, 1 << 5)] * 5
    angs = [0.4, 0.3, -0.7, 0.9] * 5
    spec = ("comp", [("coeff", 1e-6), ("weight", 6)])
    v = oracle_from_terms(N, terms, append_factor=0.2, min_capacity=4)
    g = gpu_from_oracle(v, N, append_cap=v.append_cap)
    _, ctr = v.evolve(gens, angs, window=1, strict=filt(spec), nwin=len(gens))
    wc = pp.WindowCounters(len(gens))
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(spec), counters=wc)
    assert ctr[3].sum() > 0
    assert np.array_equal(wc.terms_created, ctr[0])
    assert np.array_equal(wc.merge_in, ctr[1])
    assert np.array_equal(wc.merge_out, ctr[2])
    assert np.array_equal(wc.early_merges, ctr[3])
    assert np.all(wc.t_rotate > 0) and np.all(wc.t_merge > 0)
    compare(g, v, bitexact=True)
