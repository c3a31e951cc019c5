"""Batched instances (pp_evolve_batch) against independent oracle runs.

Each instance of a batch must equal, bit for bit, the reference's sequence
evolve! of that instance alone (spv_evolve.jl:312-387) at window = 1 with an
append capacity large enough that no early merge happens, followed by the
layer's channel: surviving key sets bit-exact, coefficients bit-identical,
<0|O_i|0> within 1e-12 * sum_{x=0}|c|."""
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import CHANNEL_KIND, filt, rand_terms, strategy

pytestmark = pytest.mark.gpu

BIG_APPEND = 1 << 20   # oracle append capacity: no early merges


def chain_layer(nq):
    gens = [((1 << (i - 1)) | (1 << i), 0) for i in range(1, nq)] + [(0, 1 << (q - 1)) for q in range(1, nq + 1)]
    acol = [0] * (nq - 1) + [1] * nq
    return gens, acol


def random_observable(rng, nq, nterms):
    obs = {}
    while len(obs) < nterms:
        w = 1 + rng.randrange(3)
        z = x = 0
        for s in rng.sample(range(nq), w):
            t = rng.randrange(3)
            if t in (0, 1):
                x |= 1 << s
            if t in (1, 2):
                z |= 1 << s
        obs[(z, x)] = rng.uniform(-1.0, 1.0)
    return [(k[0], k[1], c) for k, c in obs.items()]


def oracle_instance(nq, obs, gens, acol, ang, depth, spec, channel):
    v = orc.OracleSPV(nq, max(16, 2 * len(obs)), BIG_APPEND)
    v.upload([t[0] for t in obs], [t[1] for t in obs], [t[2] for t in obs])
    angles = [ang[a] for a in acol]
    for _ in range(depth):
        v.evolve(gens, angles, window=1, strict=filt(spec))
        if channel is not None:
            v.channel(CHANNEL_KIND[channel[0]], [channel[1]])
    return v


def run_batch(nq, ninst, depths, spec, channel, seed, keep_finished=True, nterms=3):
    rng = random.Random(seed)
    gens, acol = chain_layer(nq)
    obs = [random_observable(rng, nq, nterms) for _ in range(ninst)]
    angs = [[rng.uniform(0.05, 0.6), rng.uniform(0.05, 0.6)] for _ in range(ninst)]
    L = len(gens)
    D = max(depths)
    res = pp.evolve_batch(obs, gens * D, acol * D, angs, [d * L for d in depths], nq=nq,
                          truncation=strategy(spec),
                          channel=None if channel is None else (channel[0], channel[1], None),
                          channel_every=L, keep_finished=keep_finished)
    oracles = [oracle_instance(nq, obs[i], gens, acol, angs[i], depths[i], spec, channel) for i in range(ninst)]
    return res, oracles


@pytest.mark.parametrize("spec,channel", [
    (("coeff", 1e-6), ("depolarizing", 2e-3)),
    (("comp", [("coeff", 1e-7), ("weight", 5)]), ("dephasing", 1e-3)),
    (("comp", [("coeff", 1e-6), ("majorana", 8)]), None),
])
def test_batch_matches_independent_runs(spec, channel):
    depths = [3, 0, 1, 4, 2, 4, 1]
    res, oracles = run_batch(10, len(depths), depths, spec, channel, seed=17)
    z, x, c = res.vector.to_arrays()
    parts = pp.split_instances(z, x, c, len(depths))
    for i, v in enumerate(oracles):
        oz, ox, oc = v.arrays()
        gz, gx, gc = parts[i]
        assert np.array_equal(gz, oz[:, 0]) and np.array_equal(gx, ox[:, 0]), f"instance {i}: key sets differ"
        assert np.array_equal(gc.view(np.uint64), oc.view(np.uint64)), f"instance {i}: coefficients differ"
        assert res.n_final[i] == len(v)
        diag = ox[:, 0] == 0
        bound = 1e-12 * max(1e-300, float(np.abs(oc[diag]).sum()))
        assert abs(res.expect[i] - v.expect(0)) <= bound
    pp.check_spv(res.vector)
    assert res.stats["terms_in"] > 0


def test_batch_harvest_removes_finished():
    depths = [2, 5, 1, 3, 5, 0]
    spec = ("coeff", 1e-6)
    kept, oracles = run_batch(8, len(depths), depths, spec, ("depolarizing", 1e-3), seed=3)
    res, _ = run_batch(8, len(depths), depths, spec, ("depolarizing", 1e-3), seed=3, keep_finished=False)
    assert res.vector is None
    assert np.array_equal(res.n_final, kept.n_final)
    assert np.array_equal(res.expect.view(np.uint64), kept.expect.view(np.uint64))
    order = np.argsort(depths, kind="stable")
    t = res.t_done[order]
    assert np.all(np.diff(t) >= 0.0)
    # removing finished instances leaves less work for the later rotations
    assert res.stats["terms_in"] < kept.stats["terms_in"]


def test_batch_many_instances_large():
    """64 instances of a 12-qubit chain, uneven depths; exercises many merge tiles."""
    rng = random.Random(5)
    depths = [rng.randrange(1, 7) for _ in range(64)]
    res, oracles = run_batch(12, 64, depths, ("coeff", 1e-7), ("depolarizing", 1e-3), seed=23, nterms=4)
    for i, v in enumerate(oracles):
        assert res.n_final[i] == len(v)
        oz, ox, oc = v.arrays()
        diag = ox[:, 0] == 0
        assert abs(res.expect[i] - v.expect(0)) <= 1e-12 * max(1e-300, float(np.abs(oc[diag]).sum()))
    assert res.stats["peak"] > 20000


def test_batch_lattice64_instances():
    """Instances of the 8x8 lattice (N = 64, the whole instance word) for one layer."""
    insts = pp.circuits.batch_instances(count=5, seed=5)
    layer = [(p.z, p.x) for p in insts[0].layer]
    acol = [0] * 112 + [1] * 64
    angs = [[w.angles[0], w.angles[-1]] for w in insts]
    obs = [w.observable for w in insts]
    spec = ("coeff", 1e-4)
    res = pp.evolve_batch(obs, layer, acol, angs, [176] * 5, nq=64, truncation=strategy(spec), keep_finished=True)
    z, x, c = res.vector.to_arrays()
    parts = pp.split_instances(z, x, c, 5)
    for i in range(5):
        v = orc.OracleSPV(64, 16, BIG_APPEND)
        v.upload([t[0] for t in obs[i]], [t[1] for t in obs[i]], [t[2] for t in obs[i]])
        v.evolve(layer, [angs[i][a] for a in acol], window=1, strict=filt(spec))
        oz, ox, oc = v.arrays()
        assert np.array_equal(parts[i][0], oz[:, 0]) and np.array_equal(parts[i][1], ox[:, 0])
        assert np.array_equal(parts[i][2].view(np.uint64), oc.view(np.uint64))


def test_batch_argument_errors():
    gens, acol = chain_layer(6)
    obs = [[(1, 0, 1.0)]]
    with pytest.raises(pp.ArgumentError):
        pp.evolve_batch(obs, gens, acol, [[0.1, 0.2]], [len(gens) + 1], nq=6)
    with pytest.raises(pp.ArgumentError):
        pp.evolve_batch(obs, gens + [(1 << 7, 0)], acol + [0], [[0.1, 0.2]], [1], nq=6)
    with pytest.raises(pp.ArgumentError):
        pp.evolve_batch(obs, gens, [2] * len(gens), [[0.1, 0.2]], [1], nq=6)
    v = pp.SparsePauliVector(8, 16)
    b = pp._lib.PPBatch()
    with pytest.raises(pp.ArgumentError):
        pp._lib.check(pp._lib.lib.pp_evolve_batch(v._h, None, None, 0, b, None))
