"""pp_compact_static, the no-allocation clip entry point, against pp_compact.

A caller whose device memory belongs to another allocator (or that may not
allocate where it calls) cannot hold a pp_spv handle; pp_compact_static clips
term arrays that caller already owns, using only a static scratch array inside
the library.  This test gives it device arrays allocated by the test itself and
checks two calls in a row — the second reuses the scratch the first one left
behind — against the handle-based pp_compact on the same terms: identical keys
and bit-identical coefficients (the same per-term predicate decides; nothing is
summed), and against the CPU oracle's _compact_spv! restatement.  The filters
cover every criterion of should_drop: coefficient, weight, X weight, Majorana
weight and both exponentially damped thresholds, for one- and two-word keys.
Collected last so that a failure here never hides the other tests.
"""
import ctypes
import random

import numpy as np
import pytest

import orc
import pauliprop as pp
from helpers import filt, rand_terms, strategy
from pauliprop import _lib

pytestmark = pytest.mark.gpu


def _reference_clip(N, z, x, c, spec):
    g = pp.SparsePauliVector(N, max(16, len(c)), 16)
    g.upload(z, x, c, sorted=True)
    pp.truncate_(g, strategy(spec))
    return g.to_arrays()


def _static_clip(N, z, x, c, spec):
    import torch
    dev = torch.device("cuda", 0)
    n = len(c)
    dz = torch.from_numpy(z.view(np.int64).reshape(-1).copy()).to(dev)
    dx = torch.from_numpy(x.view(np.int64).reshape(-1).copy()).to(dev)
    dc = torch.from_numpy(c.copy()).to(dev)
    oz = torch.empty_like(dz)
    ox = torch.empty_like(dx)
    oc = torch.empty_like(dc)
    f = _lib.PPFilter(*pp.compile_filter(strategy(spec)))
    nout = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    _lib.check(_lib.lib.pp_compact_static(N, dz.data_ptr(), dx.data_ptr(), dc.data_ptr(), n, ctypes.byref(f),
                                          oz.data_ptr(), ox.data_ptr(), oc.data_ptr(), ctypes.byref(nout), None))
    m = nout.value
    nw = pp.nwords(N)
    rz = oz.cpu().numpy().view(np.uint64).reshape(-1, nw)[:m]
    rx = ox.cpu().numpy().view(np.uint64).reshape(-1, nw)[:m]
    return rz, rx, oc.cpu().numpy()[:m]


@pytest.mark.parametrize("N,n", [(64, 300_000), (100, 120_000)])
def test_static_clip_matches_handle_clip_twice(N, n):
    rng = random.Random(N)
    terms = rand_terms(rng, N, n)
    keys = sorted(terms)
    z, x = pp.pack_keys(N, keys)
    c = np.array([terms[k] for k in keys])
    for spec in (("comp", [("coeff", 0.2), ("weight", (3 * N) // 4)]), ("coeff", 0.35)):   # two calls in a row
        rz, rx, rc = _reference_clip(N, z, x, c, spec)
        sz, sx, scf = _static_clip(N, z, x, c, spec)
        assert 0 < len(rc) < n
        assert np.array_equal(sz, rz) and np.array_equal(sx, rx)
        assert np.array_equal(scf.view(np.uint64), rc.view(np.uint64))


def _oracle_clip(N, z, x, c, spec):
    v = orc.OracleSPV(N, max(16, len(c)), 16)
    v.upload(z, x, c)
    v.compact(filt(spec))
    return v.arrays()


@pytest.mark.parametrize("N", [40, 128])
def test_static_clip_every_criterion(N):
    """Every should_drop criterion (spv_kernels.jl:64-79) through the static entry
    point, two calls in a row per filter, against pp_compact and the oracle."""
    rng = random.Random(1000 + N)
    terms = rand_terms(rng, N, 50_000)
    keys = sorted(terms)
    z, x = pp.pack_keys(N, keys)
    c = np.array([terms[k] for k in keys])
    aw, axw = 1.5 / (0.75 * N), 2.0 / N         # typical weight 3N/4 and X weight N/2 of random strings
    specs = [("majorana", N), ("xweight", N // 2), ("wdamped", aw, 0.05), ("xwdamped", axw, 0.05),
             ("comp", [("coeff", 0.05), ("majorana", N + 8), ("wdamped", aw, 0.02)])]
    for spec in specs:
        rz, rx, rc = _reference_clip(N, z, x, c, spec)
        oz, ox, oc = _oracle_clip(N, z, x, c, spec)
        assert np.array_equal(rz, oz) and np.array_equal(rx, ox)
        assert 0 < len(rc) < len(c), spec
        for _ in range(2):
            sz, sx, scf = _static_clip(N, z, x, c, spec)
            assert np.array_equal(sz, oz) and np.array_equal(sx, ox), spec
            assert np.array_equal(scf.view(np.uint64), oc.view(np.uint64)), spec
            assert np.array_equal(scf.view(np.uint64), rc.view(np.uint64)), spec


def test_static_clip_rejects_oversize():
    f = _lib.PPFilter(*pp.compile_filter(pp.CoeffTruncation(0.1)))
    nout = ctypes.c_int64()
    dummy = ctypes.c_void_p(1)
    st = _lib.lib.pp_compact_static(64, dummy, dummy, dummy, (1 << 25) + 1, ctypes.byref(f),
                                    dummy, dummy, dummy, ctypes.byref(nout), None)
    assert st == _lib.PP_ARGUMENT_ERROR
    assert b"PP_COMPACT_STATIC_MAX_TERMS" in _lib.lib.pp_last_error()
