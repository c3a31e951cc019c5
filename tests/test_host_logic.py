"""Host-side logic: strategy compilation (spv_kernels.jl:81-125), Pauli strings,
qubit masks, and the seeded workload generators."""
import math

import pytest

import pauliprop as pp
from pauliprop import circuits
from pauliprop.paulis import INT64_MAX


def test_compile_filters():
    assert pp.compile_filter(pp.NoTruncation()) == pp.NOFILTER
    f = pp.compile_filter(pp.CompositeTruncation(pp.CoeffTruncation(1e-5), pp.WeightTruncation(12)))
    assert f.thresh == 1e-5 and f.wmax == 12 and f.xwmax == INT64_MAX and f.dthresh_w < 0
    f = pp.compile_filter(pp.CompositeTruncation(pp.WeightDampedTruncation(0.5, 1e-3),
                                                 pp.XWeightDampedTruncation(0.2, 1e-4), pp.WeightTruncation(4)))
    assert (f.alpha_w, f.dthresh_w, f.alpha_xw, f.dthresh_xw, f.wmax) == (0.5, 1e-3, 0.2, 1e-4, 4)
    with pytest.raises(RuntimeError):
        pp.combine_filters(pp.compile_filter(pp.WeightDampedTruncation(0.5)),
                           pp.compile_filter(pp.WeightDampedTruncation(0.6)))
    assert pp.is_compilable(pp.CompositeTruncation(pp.WeightTruncation(2), pp.CoeffTruncation(1e-4)))
    assert not pp.is_compilable(pp.AdaptiveTruncation(10, 1e-12))
    assert not pp.is_compilable(pp.CompositeTruncation(pp.WeightDampedTruncation(0.5), pp.WeightDampedTruncation(0.1)))
    assert not pp.is_compilable(pp.StochasticCoeffTruncation(0.1))


def test_default_constructors():
    # test_truncation.jl:347-355
    assert pp.CoeffTruncation().thresh == 1e-6
    assert pp.WeightDampedTruncation(0.5).thresh == 1e-6
    assert pp.XWeightDampedTruncation(0.5).alpha == 0.5
    assert pp.AdaptiveTruncation(max_terms=100, min_thresh=1e-6).max_terms == 100
    assert isinstance(pp.CompositeTruncation([pp.NoTruncation(), pp.CoeffTruncation(0.1)]).strategies, tuple)


def test_pauli_strings():
    b = pp.PauliBasis.from_string("XYZI")
    assert (b.z, b.x) == (0b0110, 0b0011)
    assert str(b) == "XYZI"
    assert pp.PauliBasis.from_sites(4, X=[1], Y=[2], Z=[3]) == b
    with pytest.raises(ValueError):
        pp.PauliBasis.from_string("XQ")


def test_qubit_mask():
    assert pp.qubit_mask(3, None) == 0b111
    assert pp.qubit_mask(3, [1, 3]) == 0b101
    assert pp.qubit_mask(3, 2) == 0b010
    for bad in ([0], [4], 4):
        with pytest.raises(pp.ArgumentError):
            pp.qubit_mask(3, bad)


def test_workloads():
    w1 = circuits.chain20()
    assert w1.N == 20 and w1.rotations == 8 * 39 and w1.observable == [(1 << 9, 0, 1.0)]
    w2 = circuits.lattice64()
    assert w2.rotations == 20 * 176 and len(w2.observable) == 64 and w2.wmax == 12
    assert len(circuits.lattice_edges()) == 112
    w3 = circuits.random_graph127()
    edges = w3.meta["edges"]
    assert len(edges) == 144 and w3.rotations == 24 * 271
    deg = {}
    for i, j in edges:
        deg[i] = deg.get(i, 0) + 1
        deg[j] = deg.get(j, 0) + 1
    assert max(deg.values()) <= 3
    assert all(0.1 <= a <= 0.5 for a in w3.angles[:144]) and all(0 <= a <= math.pi / 4 for a in w3.angles[144:])
    assert circuits.random_graph127().angles == w3.angles  # deterministic seed
    b = circuits.batch_instances(16)
    assert all(4 <= x.layers <= 24 for x in b)
    assert all(1 <= bin(x.observable[0][0] | x.observable[0][1]).count("1") <= 4 for x in b)


def test_splitmix_reference_values():
    # splitmix64 seeded with 0: published first outputs
    r = circuits.SplitMix64(0)
    assert r.next_u64() == 0xE220A8397B1DCDAF
    assert r.next_u64() == 0x6E789E6AA1B965F4


def test_trotterize_order2():
    terms = circuits.heisenberg_chain_terms(4)
    g, a = circuits.trotterize(terms, 0.1, n_trotter=2, order=2)
    assert len(g) == 2 * 2 * len(terms)
    assert g[len(terms)] == terms[-1][0] and a[0] == pytest.approx(0.05 * terms[0][1])


def test_tuning_cache_lookup(tmp_path, monkeypatch):
    """The autotuner's cache is keyed by SM count and compute capability, per word count."""
    import json
    from pauliprop import tune
    monkeypatch.setattr(tune, "TUNING_DIR", str(tmp_path))
    tune._cache.clear()
    assert tune.cached(148, 10, 0, 1) is None
    (tmp_path / "sm148_cc100.json").write_text(json.dumps(
        {"sm_count": 148, "cc": [10, 0], "nw": {"1": {"tuning": [1024, 4, 5, 64], "terms_per_s": 1.0}}}))
    tune._cache.clear()
    assert tune.cached(148, 10, 0, 1) == (1024, 4, 5, 64)
    assert tune.cached(148, 10, 0, 2) is None
    assert tune.cached(132, 9, 0, 1) is None
    tune._cache.clear()


def test_shard_owner_host_side():
    """pp_shard_owner (host-side): rank_bits GF(2)-linear parities of the key, so
    owner(P xor M) = owner(P) xor owner(M) for one- and two-word keys, every rank
    receives keys, and bad arguments are refused."""
    import numpy as np
    from pauliprop import _lib, shard
    rng = np.random.default_rng(3)
    for nw in (1, 2):
        z = rng.integers(0, 2**63, size=(4000, nw), dtype=np.uint64)
        x = rng.integers(0, 2**63, size=(4000, nw), dtype=np.uint64)
        mz = rng.integers(0, 2**63, size=(1, nw), dtype=np.uint64)
        mx = rng.integers(0, 2**63, size=(1, nw), dtype=np.uint64)
        for rb in (0, 1, 3):
            o = shard.owners(nw, z, x, rb)
            om = shard.owners(nw, mz, mx, rb)[0]
            assert np.array_equal(shard.owners(nw, z ^ mz, x ^ mx, rb), o ^ om)
            assert set(np.unique(o)) == set(range(1 << rb))
    out = np.zeros(1, dtype=np.int32)
    assert _lib.lib.pp_shard_owner(3, out.ctypes.data, out.ctypes.data, 1, 1, out.ctypes.data) == _lib.PP_ARGUMENT_ERROR
    assert _lib.lib.pp_shard_owner(1, out.ctypes.data, out.ctypes.data, 1, 9, out.ctypes.data) == _lib.PP_ARGUMENT_ERROR


def test_generator_words_and_angles_host_side():
    """evolve_'s host packing of generators into little-endian key words and its
    cos/sin of the angles (libm once per distinct angle bit pattern) equal a
    per-element restatement bit for bit: one- and two-word keys, (z, x) pairs
    mixed with PauliBasis, words beyond the key width (masked for two-word keys,
    refused for one-word keys), -0.0 against 0.0, NaN, subnormals.  No GPU
    call."""
    import random
    import numpy as np
    from pauliprop import spv
    from pauliprop.paulis import PauliBasis

    def words(N, gens):
        nw = pp.nwords(N)
        m = (1 << 64) - 1
        zs = [g.z if isinstance(g, PauliBasis) else int(g[0]) for g in gens]
        xs = [g.x if isinstance(g, PauliBasis) else int(g[1]) for g in gens]
        gz = np.array([[(z >> (64 * w)) & m for w in range(nw)] for z in zs], dtype=np.uint64).reshape(len(gens), nw)
        gx = np.array([[(x >> (64 * w)) & m for w in range(nw)] for x in xs], dtype=np.uint64).reshape(len(gens), nw)
        return gz, gx

    rng = random.Random(7)
    for N in (1, 20, 64, 65, 127, 128):
        m = (1 << N) - 1
        for L in (0, 1, 40, 700):
            gens = [PauliBasis(N, rng.getrandbits(N) & m, rng.getrandbits(N) & m) for _ in range(L)]
            cases = [gens, [((g.z, g.x) if i % 3 == 0 else g) for i, g in enumerate(gens)]]
            big = gens[:-1] + [PauliBasis(N, 1 << (64 * pp.nwords(N) + 3), 5)]
            if L and pp.nwords(N) > 1:
                cases.append(big)           # masked to the key width, as before
            elif L:
                with pytest.raises(OverflowError):
                    spv._gen_words(N, big)  # a one-word key does not fit: refused, as before
            for g2 in cases:
                a, b = words(N, g2), spv._gen_words(N, g2)
                for p, q in zip(a, b):
                    assert q.dtype == np.uint64 and q.shape == p.shape and np.array_equal(p, q)
    base = [0.3, -1.1, 2.5, 0.0, -0.0, float("nan"), 5e-324, -1e-300]
    for L in (0, 3, 16, 17, 400):
        for angles in ([rng.choice(base) for _ in range(L)], [rng.uniform(-4, 4) for _ in range(L)],
                       np.array([rng.choice(base) for _ in range(L)], dtype=np.float32)):
            c, s = spv._cos_sin(angles)
            al = np.asarray(angles, dtype=np.float64).tolist()
            assert np.array_equal(c.view(np.uint64), np.array([math.cos(a) for a in al], dtype=np.float64).view(np.uint64))
            assert np.array_equal(s.view(np.uint64), np.array([math.sin(a) for a in al], dtype=np.float64).view(np.uint64))
    with pytest.raises(ValueError):
        spv._cos_sin([0.5] * 20 + [float("inf")])


def test_batch_tags_and_shard_split_host_side():
    """Host helpers around the device calls: tagged_terms / split_instances
    round-trip each instance's terms (instance index in z word 1); shard.split
    partitions a term set exactly by owner; bits_for gives the fewest bucket
    bits whose mean load stays within cap / load_div.  No GPU call."""
    import random
    import numpy as np
    from pauliprop import shard
    from pauliprop.batch import split_instances, tagged_terms

    rng = random.Random(3)
    obs = [[(rng.getrandbits(64), rng.getrandbits(64), rng.uniform(-1, 1)) for _ in range(rng.randrange(0, 7))]
           for _ in range(5)]
    z, x, c = tagged_terms(obs)
    assert z.shape == (sum(map(len, obs)), 2) and np.array_equal(np.unique(z[:, 1]), [i for i, o in enumerate(obs) if o])
    for i, (pz, px, pc) in enumerate(split_instances(z, x, c, len(obs))):
        assert [(int(a), int(b), float(v)) for a, b, v in zip(pz, px, pc)] == obs[i]

    for nw, rank_bits in ((1, 1), (1, 3), (2, 2)):
        n = 500
        z = np.array([[rng.getrandbits(64) for _ in range(nw)] for _ in range(n)], dtype=np.uint64)
        x = np.array([[rng.getrandbits(64) for _ in range(nw)] for _ in range(n)], dtype=np.uint64)
        c = np.arange(n, dtype=np.float64)
        parts = shard.split(nw, z, x, c, rank_bits)
        assert len(parts) == 1 << rank_bits
        assert sorted(np.concatenate([p[2] for p in parts]).tolist()) == c.tolist()
        for r, (pz, px, pc) in enumerate(parts):
            assert np.all(shard.owners(nw, pz, px, rank_bits) == r)
            assert np.array_equal(pz, z[pc.astype(int)]) and np.array_equal(px, x[pc.astype(int)])

    for n in (0, 1, 1000, 10**6, 10**9):
        b = shard.bits_for(n, 512, 6)
        assert 1 <= b <= 26
        assert b == 26 or (512 << b) >= 6 * n
        assert b == 1 or (512 << (b - 1)) < 6 * n
