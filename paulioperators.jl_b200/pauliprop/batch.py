"""Batched instances: many independent SparsePauliVectors evolved in one pass.

Every instance is an nq-qubit (nq <= 64) vector with its own observable, its own
angles and its own depth (a prefix of one shared generator sequence).  They share
one GPU handle of 128-bit words: instance i's terms carry i in z word 1, so each
instance is a contiguous sorted run and every rotation kernel processes all of
them in one launch (pp_evolve_batch in include/pauliprop.h).  Instance by
instance the result equals evolve!(v_i, gens[1:rot_end[i]], angles_i;
truncation) (spv_evolve.jl:312-387) at window = 1 without early merges, with the
optional channel after every `channel_every` rotations the instance runs.
"""
import ctypes
import math
from ctypes import byref, c_double

import numpy as np

from . import _lib
from ._lib import ArgumentError, PPBatch, PPEvolveOpts, check, lib
from .paulis import PauliBasis
from .spv import CHANNEL_KINDS, SparsePauliVector, _pp_filter, _ptr
from .truncation import NoTruncation, compile_filter, is_compilable

M64 = (1 << 64) - 1


class BatchResult:
    """expect[i] = <ket|O_i|ket> after instance i's last rotation; t_done[i] = device
    seconds from the call's start until that value was ready; n_final[i] = its term
    count then; stats = the run statistics (as evolve_'s `stats`); vector = the
    batch vector when keep_finished=True (else None)."""

    def __init__(self, expect, t_done, n_final, stats, vector):
        self.expect, self.t_done, self.n_final, self.stats, self.vector = expect, t_done, n_final, stats, vector


def tagged_terms(observables):
    """Term arrays of the batch vector: observables[i] = [(z, x, c), ...] of
    instance i (nq-qubit integers) -> z, x of shape (n, 2) and c."""
    rows = [(int(z) & M64, i, int(x) & M64, float(c)) for i, obs in enumerate(observables) for z, x, c in obs]
    n = len(rows)
    z = np.zeros((n, 2), dtype=np.uint64)
    x = np.zeros((n, 2), dtype=np.uint64)
    c = np.zeros(n, dtype=np.float64)
    for r, (zl, i, xl, cv) in enumerate(rows):
        z[r, 0], z[r, 1], x[r, 0], c[r] = zl, i, xl, cv
    return z, x, c


def split_instances(z, x, c, ninst):
    """Per-instance (z, x, c) (word 0 only) of downloaded batch-vector arrays."""
    tag = z[:, 1]
    out = []
    for i in range(ninst):
        m = tag == i
        out.append((z[m, 0].copy(), x[m, 0].copy(), c[m].copy()))
    return out


def evolve_batch(observables, generators, acol, angles, rot_end, *, nq, truncation=None,
                 channel=None, channel_every=0, ket=0, keep_finished=False, profile=False,
                 capacity=None, vector=None):
    """Evolve len(observables) instances through prefixes of `generators`.

    generators: L nq-qubit generators (PauliBasis or (z, x)); acol[r]: angle column
    of rotation r; angles[i][j]: θ of instance i's column j; rot_end[i]: rotations
    instance i runs.  channel=(kind, params, qubits or None) after every
    `channel_every` rotations (0: after the last rotation).  `vector`: an existing
    SparsePauliVector(128, ...) to run in (it is overwritten and kept open)."""
    ninst = len(observables)
    if ninst < 1:
        raise ArgumentError("need at least one instance")
    L = len(generators)
    ang = np.asarray(angles, dtype=np.float64).reshape(ninst, -1)
    ncol = ang.shape[1]
    acol = np.ascontiguousarray(acol, dtype=np.int32)
    rend = np.ascontiguousarray(rot_end, dtype=np.int64)
    if len(acol) != L or len(rend) != ninst:
        raise ArgumentError("acol needs one entry per generator and rot_end one per instance")
    truncation = truncation or NoTruncation()
    if not is_compilable(truncation):
        raise NotImplementedError(f"{type(truncation).__name__} has no batched GPU path")
    cosv = np.ascontiguousarray([[math.cos(a) for a in row] for row in ang.tolist()], dtype=np.float64)
    sinv = np.ascontiguousarray([[math.sin(a) for a in row] for row in ang.tolist()], dtype=np.float64)
    gz = np.zeros((L, 2), dtype=np.uint64)
    gx = np.zeros((L, 2), dtype=np.uint64)
    for r, g in enumerate(generators):
        zz, xx = (g.z, g.x) if isinstance(g, PauliBasis) else (int(g[0]), int(g[1]))
        gz[r, 0], gx[r, 0] = zz & M64, xx & M64
    z, x, c = tagged_terms(observables)
    n = len(c)
    own = vector is None
    v = SparsePauliVector(128, capacity or max(4096, 4 * n), 16) if own else vector
    if v.N <= 64:
        raise ArgumentError("batched instances need a vector with 128-bit words (N > 64)")
    v.upload(z, x, c, sorted=False)
    expect = np.full(ninst, np.nan)
    t_done = np.zeros(ninst)
    n_final = np.zeros(ninst, dtype=np.int64)
    b = PPBatch()
    b.ninst, b.nq, b.ncol = ninst, int(nq), ncol
    b.acol, b.cosv, b.sinv, b.rot_end = _ptr(acol), _ptr(cosv), _ptr(sinv), _ptr(rend)
    b.keep_finished = 1 if keep_finished else 0
    b.expect_out, b.t_done, b.n_final = _ptr(expect), _ptr(t_done), _ptr(n_final)
    opts = PPEvolveOpts()
    opts.window = 1
    f = _pp_filter(compile_filter(truncation))
    opts.strict = ctypes.pointer(f)
    opts.strict_kind = 0
    opts.chan_kind = -1
    mask_w = None
    if channel is not None:
        kind, prm, qubits = channel
        opts.chan_kind = CHANNEL_KINDS[kind]
        prm = list(prm) if isinstance(prm, (list, tuple)) else [float(prm)]
        for i, p in enumerate(prm[:3]):
            opts.chan_prm[i] = float(p)
        if qubits is not None:
            m = 0
            for q in qubits:
                m |= 1 << (q - 1)
            mask_w = np.array([m & M64, 0], dtype=np.uint64)
            opts.chan_mask = _ptr(mask_w)
    opts.chan_every = int(channel_every or 0)
    ketw = np.array([int(ket) & M64, 0], dtype=np.uint64)
    opts.ket = _ptr(ketw)
    st = np.zeros(_lib.PP_STATS_LEN, dtype=np.float64)
    opts.stats_out = st.ctypes.data_as(ctypes.POINTER(c_double))
    opts.profile = 1 if profile else 0
    check(lib.pp_evolve_batch(v._h, _ptr(gz), _ptr(gx), L, byref(b), byref(opts)))
    stats = {name: float(st[i]) for name, i in _lib.STAT.items()}
    if not keep_finished and own:
        v.close()
        v = None
    return BatchResult(expect, t_done, n_final, stats, v)
