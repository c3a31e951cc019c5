"""Window-1 rotations on the hash-bucketed live set (k_bk_rotate) against the CPU
oracle, and against the sorted-merge kernels on the same inputs.

Sequences of at least 32 rotations over live sets above k_small_run's size run on
buckets.  Bar: bit-exact key sets and bit-identical coefficients (window 1: each
output sums at most two separately rounded products, so the bucketed order of
the partners cannot change a bit), per-rotation WindowCounters equal to the
oracle's (spv_evolve.jl:149-161), and <ket|O|ket> within 1e-12 * sum_{x=0}|c|.
The cases cover one- and two-word keys, one- to many-qubit generators (whose
bucket partner is another bucket or the same one), the early-merge pre-filter
(spv_evolve.jl:356-362), local truncation, channels fused at layer ends, growth
that splits the buckets in the middle of a call, and every compiled launch
variant (pp_set_tuning)."""
import ctypes
import os
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import CHANNEL_KIND, filt, rand_terms, strategy
from pauliprop import _lib

pytestmark = pytest.mark.gpu

VARIANTS = [(128, 4), (256, 4), (512, 4), (256, 8), (512, 8), (1024, 8)]


def _gens(rng, N, L):
    """One- to three-qubit rotations and dense strings (small angles).  With the
    thresholds used below the live sets stay within a few million terms."""
    gens, angs = [], []
    for _ in range(L):
        q = rng.sample(range(N), 3)
        kind = rng.randrange(6)
        if kind == 0:
            gens.append(((1 << q[0]) | (1 << q[1]), 0))                       # ZZ
        elif kind == 1:
            gens.append((0, 1 << q[0]))                                       # X
        elif kind == 2:
            gens.append((1 << q[0], 1 << q[0]))                               # Y
        elif kind == 3:
            gens.append(((1 << q[0]) | (1 << q[2]), (1 << q[1]) | (1 << q[2])))   # Z X Y
        elif kind == 4:
            gens.append((1 << q[0], 0))                                       # Z
        else:
            m = (1 << N) - 1
            gens.append((rng.getrandbits(N) & m, rng.getrandbits(N) & m))     # dense string
        angs.append(rng.uniform(0.02, 0.08) if kind == 5 else rng.uniform(-1.2, 1.2))
    return gens, angs


def _oracle(N, terms, **kw):
    return orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()], **kw)


def _gpu(v, N, tuning=None):
    z, x, c = v.arrays()
    g = pp.SparsePauliVector(N, max(16, 2 * len(c)), v.append_cap)
    g.upload(z, x, c, sorted=True)
    if tuning:
        _lib.check(_lib.lib.pp_set_tuning(g._h, ctypes.byref(_lib.PPTuning(*tuning))))
    return g


def _same(g, v):
    gz, gx, gc = g.to_arrays()
    oz, ox, oc = v.arrays()
    assert gz.shape == oz.shape, (gz.shape, oz.shape)
    assert np.array_equal(gz, oz) and np.array_equal(gx, ox), "key sets differ"
    assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64)), "coefficients not bit-identical"
    pp.check_spv(g)


def _on(path, fn):
    old = os.environ.get("PAULIPROP_WINDOW1_PATH")
    os.environ["PAULIPROP_WINDOW1_PATH"] = path
    try:
        return fn()
    finally:
        if old is None:
            del os.environ["PAULIPROP_WINDOW1_PATH"]
        else:
            os.environ["PAULIPROP_WINDOW1_PATH"] = old


@pytest.mark.parametrize("N", [30, 64, 100])
@pytest.mark.parametrize("spec", ["coeff", "comp"])
def test_bucket_random_sequences(N, spec):
    spec = ("coeff", 1e-2) if spec == "coeff" else ("comp", [("coeff", 1e-2), ("weight", 3 * N // 4 + 2)])
    rng = random.Random(7 * N)
    terms = rand_terms(rng, N, 5000)
    gens, angs = _gens(rng, N, 48)
    v = _oracle(N, terms)
    g = _gpu(v, N)
    t = _gpu(v, N)
    _, ctr = v.evolve(gens, angs, window=1, strict=filt(spec), nwin=len(gens))
    wc = pp.WindowCounters(len(gens))
    G = [pp.PauliBasis(N, a, b) for a, b in gens]
    _, e = _on("buckets", lambda: pp.evolve_(g, G, angs, truncation=strategy(spec), counters=wc,
                                             return_expectation=True))
    _same(g, v)
    assert np.array_equal(wc.terms_created, ctr[0])
    assert np.array_equal(wc.merge_in, ctr[1])
    assert np.array_equal(wc.merge_out, ctr[2])
    z, x, c = v.arrays()
    diag = np.all(x == 0, axis=1)
    assert abs(e - v.expect(0)) <= 1e-12 * max(1e-300, float(np.abs(c[diag]).sum()))
    # the sorted-merge kernels on the same input give the same vector
    _on("tiles", lambda: pp.evolve_(t, G, angs, truncation=strategy(spec)))
    _same(t, v)


@pytest.mark.parametrize("variant", VARIANTS, ids=str)
def test_bucket_every_variant(variant):
    """Every compiled (bucket capacity, items per thread) launch variant, with small
    load divisors and chunks, gives the oracle's vector bit for bit."""
    rng = random.Random(sum(variant))
    for N in (64, 90):
        terms = rand_terms(rng, N, 4000)
        gens, angs = _gens(rng, N, 40)
        spec = ("coeff", 1e-2)
        v = _oracle(N, terms)
        g = _gpu(v, N, tuning=(variant[0], variant[1], 3, 8))
        tn = _lib.PPTuning()
        _lib.check(_lib.lib.pp_get_tuning(g._h, ctypes.byref(tn)))
        assert (tn.bucket_cap, tn.items_per_thread, tn.load_div, tn.chunk) == (variant[0], variant[1], 3, 8)
        v.evolve(gens, angs, window=1, strict=filt(spec))
        _on("buckets", lambda: pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs,
                                          truncation=strategy(spec)))
        _same(g, v)


def test_tuning_argument_errors():
    g = pp.SparsePauliVector(8)
    for bad in ((384, 4, 5, 64), (1024, 4, 5, 64), (256, 4, 2, 64), (256, 4, 5, 4), (256, 4, 5, 512)):
        assert _lib.lib.pp_set_tuning(g._h, ctypes.byref(_lib.PPTuning(*bad))) == _lib.PP_ARGUMENT_ERROR


def test_bucket_early_merge_prefilter():
    """A small append capacity makes n > capacity, so rotations start with the
    early boundary that filters live terms before rotating (pre-filtered terms
    come back as new sin branches of their live partners)."""
    rng = random.Random(11)
    N = 40
    terms = rand_terms(rng, N, 6000)
    for k in list(terms)[:2000]:
        terms[k] = 1e-3 * (rng.random() - 0.5)       # below the threshold before any rotation
    gens, angs = _gens(rng, N, 40)
    spec = ("coeff", 1e-2)
    v = _oracle(N, terms, append_factor=0.05, min_capacity=4)
    g = _gpu(v, N)
    _, ctr = v.evolve(gens, angs, window=1, strict=filt(spec), nwin=len(gens))
    assert ctr[3].sum() > 0
    wc = pp.WindowCounters(len(gens))
    _on("buckets", lambda: pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs,
                                      truncation=strategy(spec), counters=wc))
    _same(g, v)
    assert np.array_equal(wc.early_merges, ctr[3])
    assert np.array_equal(wc.merge_in, ctr[1])
    assert np.array_equal(wc.merge_out, ctr[2])


@pytest.mark.parametrize("N", [50, 90])
def test_bucket_local_truncation_and_channel(N):
    rng = random.Random(3 + N)
    terms = rand_terms(rng, N, 5000)
    gens, angs = _gens(rng, N, 36)
    spec, lspec = ("comp", [("coeff", 1e-2), ("weight", 3 * N // 4 + 4)]), ("coeff", 2e-2)
    per = 12
    v = _oracle(N, terms)
    g = _gpu(v, N)
    for s in range(0, len(gens), per):
        v.evolve(gens[s:s + per], angs[s:s + per], window=1, strict=filt(spec), local=filt(lspec))
        v.channel(CHANNEL_KIND["depolarizing"], [0.01])
    _on("buckets", lambda: pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(spec),
                                      local_truncation=strategy(lspec), channel=("depolarizing", 0.01, None),
                                      channel_every=per))
    _same(g, v)


@pytest.mark.parametrize("N", [64, 120])
def test_bucket_growth_splits(N):
    """From 300 terms the set grows to ~1e6 (peak ~3e6) within one call: the
    single-CTA kernel hands over to buckets, which overflow or pass their split
    size in the middle of launched chunks."""
    rng = random.Random(N)
    terms = rand_terms(rng, N, 300)
    gens, angs = [], []
    for _ in range(40):
        i, j = rng.sample(range(12), 2)
        gens.append(((1 << i) | (1 << j), 0) if rng.random() < 0.6 else (0, 1 << i))
        angs.append(rng.uniform(0.2, 1.2))
    spec = ("coeff", 1e-3)
    v = _oracle(N, terms)
    g = _gpu(v, N)
    v.evolve(gens, angs, window=1, strict=filt(spec))
    _on("buckets", lambda: pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs, truncation=strategy(spec)))
    assert 10**6 < len(v) < 4 * 10**6
    _same(g, v)


def test_bucket_config2_whole_circuit():
    """The 8x8-lattice benchmark circuit (3,520 rotations, peak 3.9e6 terms) in one
    call on buckets, bit for bit against the oracle."""
    w = pp.circuits.lattice64()
    f = filt(("comp", [("coeff", w.thresh), ("weight", w.wmax)]))
    v = orc.OracleSPV.from_terms(w.N, w.observable)
    gens1 = [(p.z, p.x) for p in w.layer]
    for _ in range(w.layers):
        v.evolve(gens1, w.angles, window=1, strict=f)
        v.channel(CHANNEL_KIND[w.channel[0]], [w.channel[1]])
    ps = pp.PauliSum(w.N)
    for z, x, c in w.observable:
        ps[(z, x)] = c
    g = pp.SparsePauliVector.from_paulisum(ps)
    gens, angs = w.generators()
    _, e = _on("buckets", lambda: pp.evolve_(
        g, gens, angs, truncation=strategy(("comp", [("coeff", w.thresh), ("weight", w.wmax)])),
        channel=(w.channel[0], w.channel[1], None), channel_every=len(w.layer), return_expectation=True))
    _same(g, v)
    z, x, c = v.arrays()
    diag = np.all(x == 0, axis=1)
    assert abs(e - v.expect(0)) <= 1e-12 * max(1e-300, float(np.abs(c[diag]).sum()))


@pytest.mark.parametrize("spec,channel", [
    (("coeff", 1e-6), ("depolarizing", 2e-3)),
    (("comp", [("coeff", 1e-6), ("weight", 7)]), ("dephasing", 1e-3)),
])
@pytest.mark.parametrize("keep_finished", [True, False])
def test_bucket_batched_instances(spec, channel, keep_finished):
    """Batched instances on buckets: a 20-qubit chain (39 rotations per layer, so
    every span between instance ends runs on buckets), uneven depths.  Every
    instance equals its own oracle run bit for bit (keys, coefficients, final
    count, <0|O_i|0> within 1e-12 * sum|c_diag|), and the sorted-merge kernels
    give the same batch bit for bit."""
    from test_gpu_batch import BIG_APPEND, chain_layer, random_observable
    nq = 20
    depths = [1, 3, 4, 0, 2, 5, 3, 4]
    rng = random.Random(5)
    gens, acol = chain_layer(nq)
    obs = [random_observable(rng, nq, 3) for _ in depths]
    angs = [[rng.uniform(0.05, 0.5), rng.uniform(0.05, 0.5)] for _ in depths]
    L, D = len(gens), max(depths)
    assert L >= 32

    def go():
        return pp.evolve_batch(obs, gens * D, acol * D, angs, [d * L for d in depths], nq=nq,
                               truncation=strategy(spec), channel=(channel[0], channel[1], None),
                               channel_every=L, keep_finished=keep_finished)

    res = _on("buckets", go)
    til = _on("tiles", go)
    assert res.stats["bucket_rot"] > 0 and til.stats["bucket_rot"] == 0
    assert np.array_equal(res.n_final, til.n_final)
    assert np.array_equal(res.expect.view(np.uint64), til.expect.view(np.uint64))
    if keep_finished:
        parts = pp.split_instances(*res.vector.to_arrays(), len(depths))
        tparts = pp.split_instances(*til.vector.to_arrays(), len(depths))
    for i, d in enumerate(depths):
        v = orc.OracleSPV(nq, max(16, 2 * len(obs[i])), BIG_APPEND)
        v.upload([t[0] for t in obs[i]], [t[1] for t in obs[i]], [t[2] for t in obs[i]])
        for _ in range(d):
            v.evolve(gens, [angs[i][a] for a in acol], window=1, strict=filt(spec))
            v.channel(CHANNEL_KIND[channel[0]], [channel[1]])
        oz, ox, oc = v.arrays()
        assert res.n_final[i] == len(v)
        diag = ox[:, 0] == 0
        assert abs(res.expect[i] - v.expect(0)) <= 1e-12 * max(1e-300, float(np.abs(oc[diag]).sum()))
        if keep_finished:
            gz, gx, gc = parts[i]
            assert np.array_equal(gz, oz[:, 0]) and np.array_equal(gx, ox[:, 0]), f"instance {i}: key sets differ"
            assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64)), f"instance {i}: coefficients differ"
            for a, b in zip(parts[i], tparts[i]):
                assert np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))
    if keep_finished:
        pp.check_spv(res.vector)


@pytest.mark.parametrize("limit", [1 << 21, 1 << 12])
def test_bucket_layout_too_large_hands_over(limit):
    """When the next bucket layout does not fit in device memory (here: a test cap
    on its slots), the rotations done so far go back to the dense sorted set and
    the sorted-merge kernels finish the sequence -- in the middle of the call
    (2^21 slots: the set outgrows it) or from the start (2^12 slots: nothing
    fits).  Same vector as the oracle's, bit for bit, either way."""
    rng = random.Random(64)
    N = 64
    terms = rand_terms(rng, N, 600)          # grows to 1.7e6 terms
    gens, angs = [], []
    for _ in range(40):
        i, j = rng.sample(range(12), 2)
        gens.append(((1 << i) | (1 << j), 0) if rng.random() < 0.6 else (0, 1 << i))
        angs.append(rng.uniform(0.2, 1.2))
    spec = ("coeff", 1e-3)
    v = _oracle(N, terms)
    g = _gpu(v, N)
    v.evolve(gens, angs, window=1, strict=filt(spec))
    st = {}
    _lib.check(_lib.lib.pp_debug_bucket_limit(limit))
    try:
        _on("buckets", lambda: pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs,
                                          truncation=strategy(spec), stats=st))
    finally:
        _lib.check(_lib.lib.pp_debug_bucket_limit(0))
    assert len(v) > 10**6
    if limit > 1 << 12:
        assert 0 < st["bucket_rot"] < len(gens)
    else:
        assert st["bucket_rot"] == 0
    _same(g, v)
