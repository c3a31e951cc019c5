"""Key-sharded window-1 evolution (pauliprop.shard) against the CPU oracle.

R = 2 or 4 ranks run as virtual ranks on one GPU: one SparsePauliVector handle
per rank, exchanges copied between the handles (LocalGroup), so the kernels and
the protocol are the ones a multi-GPU run uses, with no kernel waiting on
another.  Bar: the union of the shards equals the oracle's vector of the
unsharded evolve! (spv_evolve.jl:312-387) bit for bit -- every output key sums
the same one or two terms -- every shard holds only keys it owns, and the sum of
the shards' <ket|O|ket> parts is within 1e-12 * sum_{x=0}|c| of the oracle's.
Cases: one- and two-word keys, one- to many-qubit generators, the early-merge
pre-filter (a small append capacity), local truncation, layer channels, and
growth that gives every rank more buckets."""
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import CHANNEL_KIND, filt, rand_terms, strategy
from pauliprop import shard

pytestmark = pytest.mark.gpu


def _gens(rng, N, L):
    gens, angs = [], []
    for _ in range(L):
        q = rng.sample(range(N), 3)
        kind = rng.randrange(5)
        if kind == 0:
            gens.append(((1 << q[0]) | (1 << q[1]), 0))
        elif kind == 1:
            gens.append((0, 1 << q[0]))
        elif kind == 2:
            gens.append(((1 << q[0]) | (1 << q[2]), (1 << q[1]) | (1 << q[2])))
        elif kind == 3:
            gens.append((1 << q[0], 1 << q[0]))
        else:
            m = (1 << N) - 1
            gens.append((rng.getrandbits(N) & m, rng.getrandbits(N) & m))
        angs.append(rng.uniform(0.02, 0.08) if kind == 4 else rng.uniform(-1.2, 1.2))
    return gens, angs


def _run(N, terms, gens, angs, spec, rank_bits, acap, lspec=None, channel=None, per=0):
    nw = pp.nwords(N)
    keys = list(terms)
    z, x = pp.pack_keys(N, keys)
    c = np.array([terms[k] for k in keys], dtype=np.float64)
    engines = []
    for r, (pz, px, pc) in enumerate(shard.split(nw, z, x, c, rank_bits)):
        v = pp.SparsePauliVector(N, max(16, 2 * len(pc)), 16)
        if len(pc):
            v.upload(pz, px, pc, sorted=False)
        engines.append(shard.GpuShard(v, rank_bits, r))
    G = [pp.PauliBasis(N, a, b) for a, b in gens]
    e, st = shard.run_sharded(engines, shard.LocalGroup(1 << rank_bits), N, G, angs, truncation=strategy(spec),
                              local_truncation=strategy(lspec) if lspec else None,
                              channel=None if channel is None else (channel[0], channel[1], None),
                              channel_every=per, append_capacity=acap)
    parts = []
    for eng in engines:
        gz, gx, gc = eng.v.to_arrays()
        assert np.all(shard.owners(nw, gz, gx, rank_bits) == eng.rank), "a shard holds a key it does not own"
        pp.check_spv(eng.v)
        parts.append((gz, gx, gc))
        eng.v.close()
    gz = np.concatenate([p[0] for p in parts]).reshape(-1, nw)
    gx = np.concatenate([p[1] for p in parts]).reshape(-1, nw)
    gc = np.concatenate([p[2] for p in parts])
    # key order: z then x, each as an integer whose last word is the most significant
    order = np.lexsort(tuple(gx[:, k] for k in range(nw)) + tuple(gz[:, k] for k in range(nw)))
    return gz[order], gx[order], gc[order], e, st


def _check(res, v):
    gz, gx, gc, e, _ = res
    oz, ox, oc = v.arrays()
    assert gz.shape == oz.shape, (gz.shape, oz.shape)
    assert np.array_equal(gz, oz) and np.array_equal(gx, ox), "key sets differ"
    assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64)), "coefficients not bit-identical"
    diag = np.all(ox == 0, axis=1)
    assert abs(e - v.expect(0)) <= 1e-12 * max(1e-300, float(np.abs(oc[diag]).sum()))


@pytest.mark.parametrize("rank_bits", [1, 2])
@pytest.mark.parametrize("N", [64, 100])
def test_shard_random_sequences(N, rank_bits):
    rng = random.Random(11 * N + rank_bits)
    terms = rand_terms(rng, N, 6000)
    gens, angs = _gens(rng, N, 40)
    spec = ("comp", [("coeff", 1e-2), ("weight", 3 * N // 4 + 2)])
    v = orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()])
    res = _run(N, terms, gens, angs, spec, rank_bits, v.append_cap)
    v.evolve(gens, angs, window=1, strict=filt(spec))
    _check(res, v)


def test_shard_early_merge_and_local_truncation():
    """A small append capacity makes the global count exceed it, so rotations
    start with the early-merge pre-filter, decided from the counts summed over
    ranks; local truncation filters sin branches on the rank that creates them."""
    rng = random.Random(5)
    N = 40
    terms = rand_terms(rng, N, 6000)
    for k in list(terms)[:2000]:
        terms[k] = 1e-3 * (rng.random() - 0.5)
    gens, angs = _gens(rng, N, 36)
    spec, lspec = ("coeff", 1e-2), ("coeff", 2e-2)
    v = orc.OracleSPV.from_terms(N, [(k[0], k[1], c) for k, c in terms.items()], append_factor=0.05, min_capacity=4)
    res = _run(N, terms, gens, angs, spec, 2, v.append_cap, lspec=lspec)
    _, ctr = v.evolve(gens, angs, window=1, strict=filt(spec), local=filt(lspec), nwin=len(gens))
    assert ctr[3].sum() > 0
    _check(res, v)
    assert res[4]["created"] == ctr[0].sum()


def test_shard_config2_layers_with_channel():
    """The 8x8-lattice benchmark circuit's first 6 layers with its depolarizing
    channel after each layer, on 4 ranks; the set grows past 10^5 terms, so every
    rank splits its buckets in step."""
    w = pp.circuits.lattice64()
    layers = 6
    spec = ("comp", [("coeff", w.thresh), ("weight", w.wmax)])
    terms = {(z, x): c for z, x, c in w.observable}
    v = orc.OracleSPV.from_terms(w.N, w.observable)
    gens1 = [(p.z, p.x) for p in w.layer]
    for _ in range(layers):
        v.evolve(gens1, w.angles, window=1, strict=filt(spec))
        v.channel(CHANNEL_KIND[w.channel[0]], [w.channel[1]])
    res = _run(w.N, terms, gens1 * layers, list(w.angles) * layers, spec, 2,
               orc.OracleSPV.from_terms(w.N, w.observable).append_cap, channel=w.channel, per=len(w.layer))
    assert len(v) > 10**5
    assert res[4]["bucket_bits"] > 2
    _check(res, v)


def test_shard_argument_errors():
    """Calls out of order or with bad sizes are refused with a status, and the
    handle stays usable."""
    import ctypes
    from pauliprop import _lib
    N = 64
    v = pp.SparsePauliVector(N, 64, 16)
    z, x = pp.pack_keys(N, [(1, 0), (2, 3), (0, 5)])
    v.upload(z, x, np.array([1.0, 0.5, -0.25]), sorted=False)
    n, part, st = ctypes.c_int64(), ctypes.c_int32(), np.zeros(5, dtype=np.int64)
    # no run in progress
    assert _lib.lib.pp_shard_send(v._h, 0, 0, None, None, None, 0, ctypes.byref(n), ctypes.byref(part)) \
        == _lib.PP_ARGUMENT_ERROR
    assert _lib.lib.pp_shard_rotate(v._h, 0, 0, st.ctypes.data) == _lib.PP_ARGUMENT_ERROR
    assert _lib.lib.pp_shard_end(v._h, None, None) == _lib.PP_ARGUMENT_ERROR
    # bad rank / bucket bits
    gz = np.array([[3]], dtype=np.uint64)
    gx = np.array([[0]], dtype=np.uint64)
    cs = np.array([0.5]), np.array([0.2])
    opts = _lib.PPEvolveOpts()
    opts.window = 1
    opts.chan_kind = -1
    mx = ctypes.c_int32()
    assert _lib.lib.pp_shard_begin(v._h, 1, 2, gz.ctypes.data, gx.ctypes.data, cs[0].ctypes.data, cs[1].ctypes.data,
                                   1, ctypes.byref(opts), 4, ctypes.byref(mx)) == _lib.PP_ARGUMENT_ERROR
    assert _lib.lib.pp_shard_begin(v._h, 1, 0, gz.ctypes.data, gx.ctypes.data, cs[0].ctypes.data, cs[1].ctypes.data,
                                   1, ctypes.byref(opts), 26, ctypes.byref(mx)) == _lib.PP_ARGUMENT_ERROR
    # the handle still works as a vector
    assert len(v) == 3
    pp.check_spv(v)
    v.close()
