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

from ._lib import PP_MLP_NPARAM, ArgumentError, PPDropSample, PPFeatureCtx, check, lib

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


def sample_terms(v, per_bin, nbins=10, lg_lo=-7.0, lg_hi=-1.0, seed=0):
    """Stratified sample of v's live terms: about 0.9 per_bin from each of nbins
    log10|c| bins over [lg_lo, lg_hi); returns (z, x, c) sorted by key."""
    cap = per_bin * nbins
    z = np.zeros(cap, dtype=np.uint64)
    x = np.zeros(cap, dtype=np.uint64)
    c = np.zeros(cap, dtype=np.float64)
    n = c_int64()
    check(lib.pp_sample_terms(v._h, nbins, lg_lo, lg_hi, per_bin, int(seed) & ((1 << 64) - 1), _fptr(z), _fptr(x),
                              _fptr(c), cap, byref(n)))
    k = n.value
    o = np.lexsort((x[:k], z[:k]))
    return z[:k][o], x[:k][o], c[:k][o]


def init_params(seed):
    """He-style initial parameters (float32), seeded."""
    import math
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0.0, math.sqrt(2.0 / 16), 64 * 16), np.zeros(64), rng.normal(0.0, math.sqrt(2.0 / 64), 64 * 64),
             np.zeros(64), rng.normal(0.0, math.sqrt(1.0 / 64), 64), np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)


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


def learned_truncate_(v, mlp, ctx, budget, sample=0, seed=0):
    """Keeps the `budget` live terms of largest predicted contribution (all of them
    when there are no more); returns the smallest kept score (-inf if none dropped).
    With sample > 0 it returns (cut, (z, x, c) of a uniform sample of up to `sample`
    dropped terms, number of dropped terms)."""
    cut = c_float()
    if not sample:
        check(lib.pp_learned_truncate(v._h, mlp._h, byref(ctx), int(budget), byref(cut), None))
        return cut.value
    z = np.zeros(sample, dtype=np.uint64)
    x = np.zeros(sample, dtype=np.uint64)
    c = np.zeros(sample, dtype=np.float64)
    ds = PPDropSample(int(sample), int(seed) & ((1 << 64) - 1), _fptr(z), _fptr(x), _fptr(c), 0, 0)
    check(lib.pp_learned_truncate(v._h, mlp._h, byref(ctx), int(budget), byref(cut), byref(ds)))
    k = ds.n
    o = np.lexsort((x[:k], z[:k]))
    return cut.value, (z[:k][o], x[:k][o], c[:k][o]), ds.n_dropped


# ----------------------------------------------------------------------------- the experiment
# Learned against plain truncation on an R x C open lattice (the 8 x 8, N = 64
# circuit by default): per layer RZZ(theta_J) on the edges (rows, then columns),
# RX(theta_h) on every site, then a depolarizing channel p = 1e-3; observable mean
# Z; weight cap 12 throughout.  Per angle draw (theta_J, theta_h):
#   reference   plain threshold t_ref at window 1,
#   plain       thresholds t > t_ref,
#   learned     plain threshold t_base per merge plus, after every layer, the
#               budget truncation to B terms by the network,
# each run timed on the GPU (the calls synchronise, so host time brackets the
# device work) with |<O> - <O>_ref| its error.

P_DEPOL = 1e-3
WMAX = 12


class Lattice:
    def __init__(self, R=8, C=8, layers=20):
        from .circuits import lattice_edges, xq, zz
        self.R, self.C, self.layers, self.N = R, C, layers, R * C
        edges = lattice_edges(R, C)
        self.gens = [zz(self.N, i, j) for (i, j) in edges] + [xq(self.N, q) for q in range(1, self.N + 1)]
        self.acol = [0] * len(edges) + [1] * self.N

    def angles(self, draw):
        return [draw[a] for a in self.acol]

    def ctx(self, layer, draw):
        return lattice_feature_ctx(self.R, self.C, layer, self.layers, draw[0], draw[1])

    def observable_vector(self, cap=1 << 20):
        from .spv import SparsePauliVector
        v = SparsePauliVector(self.N, cap, cap)
        z = np.array([[1 << q] for q in range(self.N)], dtype=np.uint64)
        x = np.zeros((self.N, 1), dtype=np.uint64)
        c = np.full(self.N, 1.0 / self.N)
        v.upload(z, x, c, sorted=True)
        return v


def angle_draws(count, seed, tj=(0.22, 0.32), th=(0.18, 0.28)):
    """Seeded (theta_J, theta_h) draws, uniform in the given ranges."""
    from .circuits import SplitMix64
    rng = SplitMix64(seed)
    return [(rng.uniform(*tj), rng.uniform(*th)) for _ in range(count)]


def _plain(t):
    from .truncation import CoeffTruncation, CompositeTruncation, WeightTruncation
    return CompositeTruncation(CoeffTruncation(t), WeightTruncation(WMAX))


def run_plain(lat, draw, thresh):
    """Plain threshold run: returns (<O>, seconds, peak terms)."""
    import time
    from .spv import evolve_
    v = lat.observable_vector()
    st = {}
    t0 = time.perf_counter()
    _, e = evolve_(v, lat.gens * lat.layers, lat.angles(draw) * lat.layers, truncation=_plain(thresh),
                   channel=("depolarizing", P_DEPOL, None), channel_every=len(lat.gens), return_expectation=True,
                   stats=st)
    dt = time.perf_counter() - t0
    v.close()
    return e, dt, st["peak"]


def coeff_truncate_(v, budget):
    """The budget truncation without the network: the reference's
    AdaptiveTruncation(budget, 0) (keep the terms above the (budget+1)-th largest
    |c|), on the device."""
    from .spv import truncate_
    from .truncation import AdaptiveTruncation
    truncate_(v, AdaptiveTruncation(int(budget), 0.0))


def run_learned(lat, draw, mlp, budget, t_base, audit=None):
    """Learned run: plain t_base per merge, budget truncation after every layer
    (mlp = None: by |c| instead of the network).  audit = dict(layers=(...),
    sample=K, bound=B, label_thresh=t): at those layers the cut's dropped
    contribution is estimated from K sampled dropped terms propagated exactly (at
    label_thresh) through the remaining layers; if its magnitude exceeds the bound
    the run reverts to plain truncation (no budget) for the remaining layers.
    Returns (<O>, seconds, peak, audit log); audit time is not counted."""
    import time
    from .spv import evolve_, expectation_value
    v = lat.observable_vector()
    plain = _plain(t_base)
    angs = lat.angles(draw)
    log = []
    peak = 0
    reverted = False
    t_audit = 0.0
    t0 = time.perf_counter()
    for L in range(lat.layers):
        st = {}
        evolve_(v, lat.gens, angs, truncation=plain, channel=("depolarizing", P_DEPOL, None), stats=st)
        peak = max(peak, st["peak"])
        if reverted or L == lat.layers - 1:
            continue
        if mlp is None:
            coeff_truncate_(v, budget)
            continue
        ctx = lat.ctx(L + 1, draw)
        if audit and (L + 1) in audit["layers"]:
            cut, (z, x, c), nd = learned_truncate_(v, mlp, ctx, budget, sample=audit["sample"], seed=L + 1)
            ta = time.perf_counter()
            est = 0.0
            if len(c):
                lab = contributions(lat, draw, z, x, c, L + 1, audit["label_thresh"])
                est = float(lab.sum()) * nd / len(c)
            t_audit += time.perf_counter() - ta
            ok = abs(est) <= audit["bound"]
            log.append({"layer": L + 1, "dropped": int(nd), "sampled": int(len(c)), "estimate": est, "ok": ok})
            reverted = not ok
        else:
            learned_truncate_(v, mlp, ctx, budget)
    e = expectation_value(v, 0)
    dt = time.perf_counter() - t0 - t_audit
    v.close()
    return e, dt, peak, {"reverted": reverted, "audits": log, "audit_seconds": t_audit}


def exact_contributions(lat, draw, z, x, c, layer, label_thresh, chunk=2048):
    """c_P <0|U_rest^dag P U_rest|0> for each term (z, x, c) present after `layer`
    layers: every term is propagated alone, as one instance of a batched run,
    through the remaining layers (channel included) at the label threshold."""
    from .batch import evolve_batch
    from .spv import SparsePauliVector
    rem = lat.layers - layer
    out = np.zeros(len(c))
    if rem == 0:
        return np.where(np.asarray(x) == 0, c, 0.0)
    v = SparsePauliVector(128, 1 << 16, 16)
    L = len(lat.gens)

    def run(lo, hi):
        obs = [[(int(z[i]), int(x[i]), float(c[i]))] for i in range(lo, hi)]
        k = hi - lo
        try:
            res = evolve_batch(obs, lat.gens * rem, lat.acol * rem, [list(draw)] * k, [rem * L] * k, nq=lat.N,
                               truncation=_plain(label_thresh), channel=("depolarizing", P_DEPOL, None),
                               channel_every=L, vector=v)
        except MemoryError:
            if k == 1:
                raise
            mid = (lo + hi) // 2      # too many live terms at once: split the batch
            run(lo, mid)
            run(mid, hi)
            return
        out[lo:hi] = res.expect

    for s in range(0, len(c), chunk):
        run(s, min(len(c), s + chunk))
    v.close()
    return out


def label_thresholds(c, base, rel=1e-3):
    """Label threshold of each term: rel x (the term's |c| rounded up to a power of
    ten), never below `base`: every term is propagated to the same relative
    precision, so small terms near the truncation cut keep their (collectively
    large) contributions and large terms do not cost more than small ones."""
    a = np.maximum(np.abs(np.asarray(c, dtype=np.float64)), 1e-300)
    return np.maximum(base, rel * 10.0 ** np.ceil(np.log10(a)))


def contributions(lat, draw, z, x, c, layer, base):
    """exact_contributions with the per-term label_thresholds (one batched run per
    distinct threshold)."""
    t = label_thresholds(c, base)
    out = np.zeros(len(c))
    for tv in np.unique(t):
        m = t == tv
        out[m] = exact_contributions(lat, draw, z[m], x[m], c[m], layer, float(tv))
    return out


def _features_of(lat, z, x, c, ctx):
    """Features of given terms (computed on the device)."""
    from .spv import SparsePauliVector
    w = SparsePauliVector(lat.N, max(16, len(c)), 16)
    w.upload(z.reshape(-1, 1), x.reshape(-1, 1), c, sorted=True)
    f = features(w, ctx)
    w.close()
    return f


def training_set(lat, draws, sample_layers, per_layer, t_base, label_thresh, seed=0):
    """Features, log10 |exact contribution| targets and the contributions of terms
    sampled from the plain t_base runs of the given draws: at each sample layer,
    about per_layer terms in equal shares from ten log10|c| bins over [-7, -1)."""
    from .spv import evolve_
    rng = np.random.default_rng(seed)
    feats, targets, labels = [], [], []
    for draw in draws:
        angs = lat.angles(draw)
        v = lat.observable_vector()
        done = 0
        for Ls in sample_layers:
            evolve_(v, lat.gens * (Ls - done), angs * (Ls - done), truncation=_plain(t_base),
                    channel=("depolarizing", P_DEPOL, None), channel_every=len(lat.gens))
            done = Ls
            z, x, c = sample_terms(v, max(1, per_layer // 10), seed=int(rng.integers(1 << 62)))
            if len(c) == 0:
                continue
            f = _features_of(lat, z, x, c, lat.ctx(Ls, draw))
            lab = contributions(lat, draw, z, x, c, Ls, label_thresh)
            feats.append(f)
            labels.append(lab)
            targets.append(np.log10(np.maximum(np.abs(lab), 1e-12)).astype(np.float32))
        v.close()
    return np.concatenate(feats), np.concatenate(targets), np.concatenate(labels)


def time_to_error(runs, tol):
    """Least time among runs [(error, seconds), ...] whose error is within tol."""
    ok = [t for e, t in runs if e <= tol]
    return min(ok) if ok else None
