"""Learned truncation: a small network that predicts how much a term will still
contribute to the final expectation value, and a budget truncation that keeps the
terms it ranks highest.

Nothing here has a counterpart in the reference (PauliOperators.jl truncates by
coefficient and weight).  The network (16 features -> 64 -> 64 -> 1, GELU) runs
and trains on the GPU's tensor cores (BF16 operands, FP32 accumulation) through
libpauliprop: `MLP.forward`, `MLP.grad`, `MLP.train`; `learned_truncate_` scores
every live term in one fused pass and keeps exactly `budget` of them (ties: the
smaller (z, x) key).  Plain threshold truncation stays the fallback: the driver
in `evolve_learned` audits the learned cut and reverts to plain truncation when
its estimated error exceeds the stated bound.
"""
import ctypes
from ctypes import byref, c_float, c_int64, c_void_p

import numpy as np

from ._lib import PP_MLP_NPARAM, ArgumentError, PPFeatureCtx, check, lib

NFEAT = 16
NPARAM = PP_MLP_NPARAM


def _fptr(a):
    return a.ctypes.data_as(c_void_p)


def lattice_feature_ctx(R, C, layer, layers, theta_j, theta_h, light_cone=None):
    """Feature context of an R x C open lattice (qubit q = C*r + c + 1 is bit C*r + c)
    after `layer` of `layers` layers, for a circuit with angles theta_j, theta_h.
    light_cone: qubit mask of the remaining circuit's light cone (default: all)."""
    n = R * C
    if n > 64:
        raise ArgumentError("term features need N <= 64")
    ctx = PPFeatureCtx()
    ctx.nq = n
    full = (1 << n) - 1 if n < 64 else (1 << 64) - 1
    bnd = 0
    for r in range(R):
        for c in range(C):
            q = C * r + c
            m = 0
            for dr, dc in ((-1, 0), (1, 0), (0, -1), (0, 1)):
                rr, cc = r + dr, c + dc
                if 0 <= rr < R and 0 <= cc < C:
                    m |= 1 << (C * rr + cc)
            ctx.nbr[q] = m
            ctx.row[q] = r
            ctx.col[q] = c
            if r in (0, R - 1) or c in (0, C - 1):
                bnd |= 1 << q
    ctx.light_cone = full if light_cone is None else int(light_cone) & full
    ctx.boundary = bnd
    ctx.layer_frac = layer / layers
    ctx.remaining_frac = (layers - layer) / layers
    ctx.theta_j = theta_j
    ctx.theta_h = theta_h
    return ctx


def features(v, ctx):
    """The 16 features of every live term of v (n x 16 float32)."""
    n = c_int64()
    check(lib.pp_features(v._h, byref(ctx), None, 0, byref(n)))
    out = np.zeros((n.value, NFEAT), dtype=np.float32)
    m = c_int64()
    check(lib.pp_features(v._h, byref(ctx), _fptr(out), n.value, byref(m)))
    return out


class MLP:
    """The learned-truncation network on the GPU (FP32 master parameters, BF16 copy)."""

    def __init__(self, params=None):
        h = c_void_p()
        check(lib.pp_mlp_create(byref(h)))
        self._h = h
        if params is not None:
            self.set_params(params)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != NPARAM:
            raise ArgumentError(f"need {NPARAM} parameters")
        check(lib.pp_mlp_set_params(self._h, _fptr(p)))

    def get_params(self):
        p = np.zeros(NPARAM, dtype=np.float32)
        check(lib.pp_mlp_get_params(self._h, _fptr(p)))
        return p

    def forward(self, feat):
        feat = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, NFEAT)
        out = np.zeros(len(feat), dtype=np.float32)
        check(lib.pp_mlp_forward(self._h, _fptr(feat), len(feat), _fptr(out)))
        return out

    def grad(self, feat, target):
        feat = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, NFEAT)
        target = np.ascontiguousarray(target, dtype=np.float32)
        g = np.zeros(NPARAM, dtype=np.float32)
        loss = c_float()
        check(lib.pp_mlp_grad(self._h, _fptr(feat), _fptr(target), len(feat), _fptr(g), byref(loss)))
        return g, loss.value

    def load_data(self, feat, target):
        self._feat = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, NFEAT)
        self._target = np.ascontiguousarray(target, dtype=np.float32)
        check(lib.pp_mlp_load_data(self._h, _fptr(self._feat), _fptr(self._target), len(self._feat)))

    def train(self, steps, batch=8192, lr=1e-3, seed=0):
        """Adam steps on the loaded data; returns each step's minibatch loss."""
        losses = np.zeros(max(steps, 1), dtype=np.float32)
        check(lib.pp_mlp_train(self._h, int(steps), int(batch), float(lr), int(seed) & ((1 << 64) - 1),
                               _fptr(losses)))
        return losses[:steps]

    def close(self):
        if getattr(self, "_h", None):
            lib.pp_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def learned_truncate_(v, mlp, ctx, budget):
    """Keeps the `budget` live terms of largest predicted contribution (all of them
    when there are no more); returns the smallest kept score (-inf if none dropped)."""
    cut = c_float()
    check(lib.pp_learned_truncate(v._h, mlp._h, byref(ctx), int(budget), byref(cut)))
    return cut.value
