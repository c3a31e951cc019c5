"""Failure detection without a GPU fault (the reference models capacity exhaustion
by forcing tiny buffers, test_spv_evolution.jl:154-167, and grows and retries,
spv_evolve.jl:356-362, spv_kernels.jl:377-386).

- Allocation failure, injected on the host (pp_debug_fail_alloc): whichever
  device allocation of an evolve! call fails -- a live-set growth, the bucket
  sets, a workspace -- the call reports PP_OUT_OF_MEMORY (MemoryError) and the
  handle holds a valid vector, the oracle's after the rotations that completed;
  resumed with the remaining rotations, it ends equal to the oracle.  Both
  window-1 paths are covered.
- A bounded device wait that runs out: a look-back on a status nothing publishes
  gives up after its poll limit, the host gets PP_TIMEOUT (TimeoutError), and the
  device keeps answering."""
import os
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import filt, rand_terms, strategy
from pauliprop import _lib

pytestmark = pytest.mark.gpu


def _gens(rng, N, L):
    # rotations on 12 qubits: the set grows ~100x at threshold 1e-2 (bounded)
    gens, angs = [], []
    for _ in range(L):
        i, j = rng.sample(range(12), 2)
        gens.append(((1 << i) | (1 << j), 0) if rng.random() < 0.6 else (0, 1 << i))
        angs.append(rng.uniform(0.2, 1.2))
    return gens, angs


def _matches(g, v):
    gz, gx, gc = g.to_arrays()
    oz, ox, oc = v.arrays()
    return (gz.shape == oz.shape and np.array_equal(gz, oz) and np.array_equal(gx, ox)
            and np.array_equal(gc.view(np.uint64), oc.view(np.uint64)))


@pytest.mark.parametrize("path", ["tiles", "buckets"])
@pytest.mark.parametrize("after", [1, 2, 3, 5, 8, 13, 21, 30, 40, 50, 60])
def test_injected_allocation_failure_leaves_handle_usable(after, path):
    """The after-th device allocation of the call fails.  The call raises
    MemoryError; the handle then holds a valid vector: the oracle's vector after
    the k rotations that completed (k = 0 when the failure came before any, and
    always 0 on buckets, whose live set changes only when the sequence is done).
    Resuming with the remaining rotations gives the oracle's final vector."""
    rng = random.Random(after)
    N = 64
    terms = rand_terms(rng, N, 5000)
    keys = sorted(terms)
    z, x = pp.pack_keys(N, keys)
    c = np.array([terms[k] for k in keys])
    gens, angs = _gens(rng, N, 40)
    G = [pp.PauliBasis(N, a, b) for a, b in gens]
    spec = ("coeff", 1e-2)
    f = filt(spec)
    v = orc.OracleSPV(N, 16, 5000)
    v.upload(z, x, c)
    old = os.environ.get("PAULIPROP_WINDOW1_PATH")
    os.environ["PAULIPROP_WINDOW1_PATH"] = path
    try:
        g = pp.SparsePauliVector(N, 5000, 5000)     # room for the input only: the call must grow
        g.upload(z, x, c, sorted=True)
        _lib.check(_lib.lib.pp_debug_fail_alloc(after))
        k = len(G)
        try:
            pp.evolve_(g, G, angs, truncation=strategy(spec))
        except MemoryError as e:
            assert "injected" in str(e)
            pp.check_spv(g)
            # which prefix of the sequence the handle holds
            k = 0
            while not _matches(g, v):
                assert k < len(G), "the handle holds no state of the sequence"
                v.evolve(gens[k:k + 1], angs[k:k + 1], window=1, strict=f)
                k += 1
            if path == "buckets":
                assert k == 0
        finally:
            _lib.check(_lib.lib.pp_debug_fail_alloc(0))
        if k < len(G):
            pp.evolve_(g, G[k:], angs[k:], truncation=strategy(spec))
            v.evolve(gens[k:], angs[k:], window=1, strict=f)
        else:
            v.evolve(gens, angs, window=1, strict=f)
    finally:
        if old is None:
            del os.environ["PAULIPROP_WINDOW1_PATH"]
        else:
            os.environ["PAULIPROP_WINDOW1_PATH"] = old
    assert _matches(g, v)


def test_bounded_wait_times_out_and_device_answers():
    st = _lib.lib.pp_debug_lookback_timeout(2000)
    assert st == _lib.PP_TIMEOUT
    with pytest.raises(TimeoutError):
        _lib.check(st)
    assert _lib.lib.pp_debug_lookback_timeout(0) == _lib.PP_ARGUMENT_ERROR
    # the context is intact: a small evolve! still matches the oracle
    N = 8
    v = orc.OracleSPV.from_terms(N, [(1 << 3, 0, 1.0)])
    g = pp.SparsePauliVector(N)
    g.upload(*v.arrays(), sorted=True)
    gens = [(0b11 << k, 0) for k in range(7)] + [(0, 1 << k) for k in range(8)]
    angs = [0.3] * 7 + [0.2] * 8
    v.evolve(gens, angs, window=1)
    pp.evolve_(g, [pp.PauliBasis(N, a, b) for a, b in gens], angs)
    gz, gx, gc = g.to_arrays()
    oz, ox, oc = v.arrays()
    assert np.array_equal(gz, oz) and np.array_equal(gc.view(np.uint64), oc.view(np.uint64))
