"""GPU-resident SparsePauliVector: the reference's SPV API over libpauliprop.

Mirrors, name for name, the SparsePauliVector entry points of PauliOperators.jl
(Julia's `f!` becomes `f_`):
  SparsePauliVector(...)            type_SparsePauliVector.jl:138-188
  PauliSum(v) / to_paulisum         type_SparsePauliVector.jl:212-221
  evolve_(v, G, θ)                  spv_evolve.jl:228-236
  evolve_(v, gens, angles; ...)     spv_evolve.jl:312-387
  coeff_clip_ ... majorana_...      spv_evolve.jl:13-26
  truncate_(v, strategy, corr)      truncation.jl:330-337
  *_channel_                        channels.jl:203-265
  expectation_value(v, ket)         spv_evolve.jl:133-134
  check_spv(v)                      type_SparsePauliVector.jl:263-278
Term arrays stay in device memory between calls.
"""
import ctypes
import math
import operator
from ctypes import byref, c_double, c_int32, c_int64, c_void_p

import numpy as np

from . import _lib
from ._lib import (ArgumentError, DimensionMismatch, PPCounters, PPEvolveOpts, PPFilter,
                   check, lib)
from .paulis import PauliBasis, PauliSum, nwords, pack_keys, pack_word, qubit_mask, unpack_keys
from .truncation import (AdaptiveTruncation, CompositeTruncation, EnergyCorrection, EnergyVarianceCorrection,
                         NoCorrection, NoTruncation, StochasticCoeffTruncation, StochasticSamplingTruncation,
                         compile_filter, draw_seed, is_compilable)

CHANNEL_KINDS = {"depolarizing": 0, "dephasing": 1, "bit_flip": 2, "bit_phase_flip": 3, "pauli": 4}


def _ptr(a):
    return a.ctypes.data_as(c_void_p) if a is not None else None


def _pp_filter(f):
    return PPFilter(*f)


class WindowCounters:
    """WindowCounters(nwindows) (spv_evolve.jl:149-161)."""

    def __init__(self, nw):
        self.terms_created = np.zeros(nw, dtype=np.int64)
        self.merge_in = np.zeros(nw, dtype=np.int64)
        self.merge_out = np.zeros(nw, dtype=np.int64)
        self.early_merges = np.zeros(nw, dtype=np.int64)
        self.t_rotate = np.zeros(nw, dtype=np.float64)
        self.t_merge = np.zeros(nw, dtype=np.float64)

    def _c(self):
        P64 = ctypes.POINTER(c_int64)
        PD = ctypes.POINTER(c_double)
        return PPCounters(len(self.terms_created),
                          self.terms_created.ctypes.data_as(P64), self.merge_in.ctypes.data_as(P64),
                          self.merge_out.ctypes.data_as(P64), self.early_merges.ctypes.data_as(P64),
                          self.t_rotate.ctypes.data_as(PD), self.t_merge.ctypes.data_as(PD))


class SparsePauliVector:
    """N-qubit sum of Pauli terms with Float64 coefficients, resident on the GPU."""

    def __init__(self, N, capacity=16, append_capacity=None):
        self.N = int(N)
        self.nw = nwords(self.N)
        cap = max(int(capacity), 1)
        acap = cap if append_capacity is None else max(int(append_capacity), 1)
        h = c_void_p()
        check(lib.pp_create(self.N, cap, acap, byref(h)))
        self._h = h
        from .tune import apply_cached
        apply_cached(self)          # the autotuned launch configuration of this device, if cached

    # -- construction / conversion ------------------------------------------
    @classmethod
    def from_paulisum(cls, ps, capacity_factor=2.0, append_factor=1.0, min_capacity=16, imag_tol=1e-10):
        """SparsePauliVector(O::PauliSum; T=Float64, ...) (type_SparsePauliVector.jl:167-188)."""
        if capacity_factor < 1:
            raise ArgumentError("capacity_factor must be >= 1")
        live_cap = max(min_capacity, math.ceil(capacity_factor * max(len(ps), 1)))
        append_cap = max(min_capacity, math.ceil(append_factor * live_cap))
        keys = list(ps.keys())
        coeffs = []
        for k in keys:
            c = ps[k]
            if isinstance(c, complex):
                if abs(c.imag) > imag_tol * max(1.0, abs(c)):
                    raise _lib.PauliPropError(
                        f"coefficient {c} has an imaginary part; use a complex coefficient type "
                        "or provide Hermitian (real-coefficient) input")
                c = c.real
            coeffs.append(float(c))
        v = cls(ps.N, live_cap, append_cap)
        z, x = pack_keys(ps.N, keys)
        v.upload(z, x, np.asarray(coeffs, dtype=np.float64), sorted=False)
        return v

    @classmethod
    def from_arrays(cls, N, z, x, c, sorted=False, capacity=None, append_capacity=None):
        n = len(c)
        v = cls(N, capacity or max(16, 2 * n), append_capacity or max(16, 2 * n))
        v.upload(z, x, c, sorted=sorted)
        return v

    def upload(self, z, x, c, sorted=False):
        z = np.ascontiguousarray(z, dtype=np.uint64)
        x = np.ascontiguousarray(x, dtype=np.uint64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        n = len(c)
        if z.size != n * self.nw or x.size != n * self.nw:
            raise DimensionMismatch("z/x word arrays do not match the coefficient count")
        check(lib.pp_upload(self._h, _ptr(z), _ptr(x), _ptr(c), n, 1 if sorted else 0))

    def to_arrays(self):
        """Download (z, x, c); z, x have shape (n, nwords)."""
        n = len(self)
        z = np.zeros((n, self.nw), dtype=np.uint64)
        x = np.zeros((n, self.nw), dtype=np.uint64)
        c = np.zeros(n, dtype=np.float64)
        m = c_int64()
        check(lib.pp_download(self._h, _ptr(z), _ptr(x), _ptr(c), n, byref(m)))
        return z, x, c

    def to_paulisum(self):
        """PauliSum(v) (type_SparsePauliVector.jl:212-221)."""
        z, x, c = self.to_arrays()
        ps = PauliSum(self.N)
        for k, cv in zip(unpack_keys(z, x), c.tolist()):
            ps[k] = cv
        return ps

    def __len__(self):
        n = c_int64()
        check(lib.pp_length(self._h, byref(n)))
        return n.value

    def copy(self):
        """copy(v) (type_SparsePauliVector.jl:249-254)."""
        h = c_void_p()
        check(lib.pp_copy(self._h, byref(h)))
        o = SparsePauliVector.__new__(SparsePauliVector)
        o.N, o.nw, o._h = self.N, self.nw, h
        return o

    # -- algebra (spv_ops.jl) ----------------------------------------------------
    def __neg__(self):
        return scaled(self, -1.0)

    def __add__(self, other):
        return add(self, other)

    def __sub__(self, other):
        return sub(self, other)

    def __mul__(self, other):
        if isinstance(other, SparsePauliVector):
            return product(self, other)
        return scaled(self, other)

    def __rmul__(self, a):
        return scaled(self, a)

    def device_bytes(self):
        b = c_int64()
        check(lib.pp_device_bytes(self._h, byref(b)))
        return b.value

    def stream(self):
        s = c_void_p()
        check(lib.pp_stream(self._h, byref(s)))
        return s.value

    def close(self):
        if getattr(self, "_h", None):
            lib.pp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def PauliSum_from(v):
    return v.to_paulisum()


_get_z, _get_x = operator.attrgetter("z"), operator.attrgetter("x")


def _gen_words(N, generators):
    nw = nwords(N)
    L = len(generators)
    if nw == 1:
        try:                        # all PauliBasis (the usual case): no per-item type test
            gz = np.fromiter(map(_get_z, generators), np.uint64, L)
            gx = np.fromiter(map(_get_x, generators), np.uint64, L)
        except AttributeError:      # (z, x) pairs among them
            gz = np.fromiter((g.z if type(g) is PauliBasis else int(g[0]) for g in generators), np.uint64, L)
            gx = np.fromiter((g.x if type(g) is PauliBasis else int(g[1]) for g in generators), np.uint64, L)
        return gz.reshape(L, 1), gx.reshape(L, 1)
    nb = 8 * nw
    try:                            # all PauliBasis with in-range words: little-endian bytes of each int
        bz = b"".join([z.to_bytes(nb, "little") for z in map(_get_z, generators)])
        bx = b"".join([x.to_bytes(nb, "little") for x in map(_get_x, generators)])
        return (np.frombuffer(bz, dtype="<u8").reshape(L, nw).astype(np.uint64),
                np.frombuffer(bx, dtype="<u8").reshape(L, nw).astype(np.uint64))
    except (AttributeError, OverflowError):
        pass                        # (z, x) pairs, or words beyond nw * 64 bits (masked below)
    m = (1 << 64) - 1
    zs = [g.z if isinstance(g, PauliBasis) else int(g[0]) for g in generators]
    xs = [g.x if isinstance(g, PauliBasis) else int(g[1]) for g in generators]
    gz = np.empty((L, nw), dtype=np.uint64)
    gx = np.empty((L, nw), dtype=np.uint64)
    for w in range(nw):
        gz[:, w] = np.fromiter(((z >> (64 * w)) & m for z in zs), dtype=np.uint64, count=L)
        gx[:, w] = np.fromiter(((x >> (64 * w)) & m for x in xs), dtype=np.uint64, count=L)
    return gz, gx


def _cos_sin(angles):
    """cos θ and sin θ of every angle from the host's libm (math.cos / math.sin,
    as the reference computes them on its host, spv_evolve.jl:341-342), each
    evaluated once per distinct angle: a circuit of repeated layers has few.
    Angles are told apart by their bit patterns, so -0.0 and 0.0 (whose sines
    differ in sign) and NaN payloads are kept apart."""
    ang = angles if isinstance(angles, np.ndarray) else np.fromiter(angles, np.float64, len(angles))
    ang = np.ascontiguousarray(ang, dtype=np.float64)
    if len(ang) <= 16:
        al = ang.tolist()
        return (np.fromiter(map(math.cos, al), np.float64, len(al)),
                np.fromiter(map(math.sin, al), np.float64, len(al)))
    u, inv = np.unique(ang.view(np.uint64), return_inverse=True)
    ul = u.view(np.float64).tolist()
    cu = np.fromiter(map(math.cos, ul), np.float64, len(ul))
    su = np.fromiter(map(math.sin, ul), np.float64, len(ul))
    return cu[inv], su[inv]


def evolve_(v, G, theta=None, *, window=1, truncation=None, local_truncation=None,
            correction=None, counters=None, channel=None, channel_every=0,
            return_expectation=False, stats=None, profile=False):
    """evolve!(v, G, θ) or evolve!(v, generators, angles; window, truncation,
    local_truncation, correction, counters).

    `channel=(kind, params, qubits)` additionally applies that channel after the
    last rotation, fused into its merge (equivalent to calling the *_channel_
    function afterwards).  With `channel_every=k` the call behaves like the loop
    `for layer: evolve_(v, layer, ...); channel_(v, ...)` over consecutive
    k-rotation layers.  `stats` (a dict) receives the run statistics
    (terms_in, created, merge_in, merge_out, peak, early, launches and, with
    `profile=True`, per-kernel device seconds)."""
    if isinstance(G, PauliBasis) or (isinstance(G, tuple) and len(G) == 2 and not isinstance(G[0], PauliBasis)
                                      and theta is not None and np.ndim(theta) == 0):
        gz, gx = _gen_words(v.N, [G])
        th = float(theta)
        check(lib.pp_evolve1(v._h, _ptr(gz), _ptr(gx), math.cos(th), math.sin(th)))
        return v
    generators, angles = G, theta
    if len(generators) != len(angles):
        raise DimensionMismatch("generators and angles must have same length")
    if window < 1:
        raise ArgumentError("window must be >= 1")
    truncation = truncation or NoTruncation()
    local_truncation = local_truncation or NoTruncation()
    correction = correction or NoCorrection()
    if not is_compilable(local_truncation):
        raise ArgumentError("local_truncation must be a deterministic (weight/coefficient) "
                            "strategy — it runs per append")
    opts = PPEvolveOpts()
    opts.window = window
    strict_f = local_f = None
    if is_compilable(truncation):
        strict_f = _pp_filter(compile_filter(truncation))
        opts.strict = ctypes.pointer(strict_f)
        opts.strict_kind = 0
    elif isinstance(truncation, AdaptiveTruncation):
        opts.strict_kind = 1
        opts.adapt_max_terms = truncation.max_terms
        opts.adapt_min_thresh = truncation.min_thresh
    elif isinstance(truncation, StochasticCoeffTruncation):
        opts.strict_kind = 2
        opts.adapt_min_thresh = truncation.epsilon
        opts.seed = draw_seed(truncation.rng)
    elif isinstance(truncation, StochasticSamplingTruncation):
        opts.strict_kind = 3
        opts.adapt_max_terms = truncation.n_keep
        opts.seed = draw_seed(truncation.rng)
    else:
        raise NotImplementedError(f"{type(truncation).__name__} has no GPU path (no CPU fallback)")
    local_f = _pp_filter(compile_filter(local_truncation))
    opts.local = ctypes.pointer(local_f)
    ket = None
    ce = c_double(0.0)
    cv = c_double(0.0)
    if isinstance(correction, (EnergyCorrection, EnergyVarianceCorrection)):
        opts.corr_kind = 2 if isinstance(correction, EnergyVarianceCorrection) else 1
        ket = pack_word(v.N, correction.ket)
        opts.ket = _ptr(ket)
        ce.value = correction.accumulated_energy
        opts.corr_energy = ctypes.pointer(ce)
        if isinstance(correction, EnergyVarianceCorrection):
            cv.value = correction.accumulated_variance
            opts.corr_variance = ctypes.pointer(cv)
    elif not isinstance(correction, NoCorrection):
        raise NotImplementedError(f"{type(correction).__name__} has no GPU path (no CPU fallback)")
    cc = counters._c() if counters is not None else None
    if cc is not None:
        opts.counters = ctypes.pointer(cc)
    opts.chan_kind = -1
    mask_w = None
    if channel is not None:
        kind, prm, qubits = channel
        opts.chan_kind = CHANNEL_KINDS[kind]
        prm = list(prm) if isinstance(prm, (list, tuple)) else [float(prm)]
        for i, p in enumerate(prm[:3]):
            opts.chan_prm[i] = float(p)
        mask_w = pack_word(v.N, qubit_mask(v.N, qubits))
        opts.chan_mask = _ptr(mask_w)
    opts.chan_every = int(channel_every or 0)
    eo = c_double(float("nan"))
    opts.expect_out = ctypes.pointer(eo)
    st = np.zeros(_lib.PP_STATS_LEN, dtype=np.float64)
    opts.stats_out = st.ctypes.data_as(ctypes.POINTER(c_double))
    opts.profile = 1 if profile else 0
    gz, gx = _gen_words(v.N, generators)
    cosv, sinv = _cos_sin(angles)
    check(lib.pp_evolve(v._h, _ptr(gz), _ptr(gx), _ptr(cosv), _ptr(sinv), len(cosv), byref(opts)))
    if isinstance(correction, (EnergyCorrection, EnergyVarianceCorrection)):
        correction.accumulated_energy = ce.value
    if isinstance(correction, EnergyVarianceCorrection):
        correction.accumulated_variance = cv.value
    if stats is not None:
        for name, i in _lib.STAT.items():
            stats[name] = float(st[i])
    if return_expectation:
        return v, eo.value
    return v


def evolve(v, G, theta=None, **kw):
    """Non-mutating evolve (spv_evolve.jl:243-244, 394-396)."""
    return evolve_(v.copy(), G, theta, **kw)


def _compact(v, strategy):
    f = _pp_filter(compile_filter(strategy))
    check(lib.pp_compact(v._h, byref(f)))
    return v


def coeff_clip_(v, thresh):
    from .truncation import CoeffTruncation
    return _compact(v, CoeffTruncation(float(thresh)))


def clip_(v, thresh=1e-16):
    return coeff_clip_(v, thresh)


def weight_clip_(v, max_weight):
    from .truncation import WeightTruncation
    return _compact(v, WeightTruncation(max_weight))


def x_weight_clip_(v, max_weight):
    from .truncation import XWeightTruncation
    return _compact(v, XWeightTruncation(max_weight))


def majorana_weight_clip_(v, max_weight):
    from .truncation import MajoranaWeightTruncation
    return _compact(v, MajoranaWeightTruncation(max_weight))


def weight_damped_clip_(v, alpha, thresh):
    from .truncation import WeightDampedTruncation
    return _compact(v, WeightDampedTruncation(alpha, thresh))


def x_weight_damped_clip_(v, alpha, thresh):
    from .truncation import XWeightDampedTruncation
    return _compact(v, XWeightDampedTruncation(alpha, thresh))


def _apply_(v, s):
    """_apply! (spv_evolve.jl:59-119) for the strategies with a GPU path."""
    if isinstance(s, NoTruncation):
        return v
    if isinstance(s, CompositeTruncation):
        for x in s.strategies:
            _apply_(v, x)
        return v
    if is_compilable(s):
        return _compact(v, s)
    if isinstance(s, AdaptiveTruncation):
        check(lib.pp_adaptive(v._h, s.max_terms, s.min_thresh))
        return v
    if isinstance(s, StochasticCoeffTruncation):
        check(lib.pp_stochastic_clip(v._h, s.epsilon, draw_seed(s.rng)))
        return v
    if isinstance(s, StochasticSamplingTruncation):
        check(lib.pp_stochastic_sample(v._h, s.n_keep, draw_seed(s.rng)))
        return v
    raise NotImplementedError(f"{type(s).__name__} has no GPU path (no CPU fallback)")


def truncate_(v, strategy, corr=None):
    """truncate!(O, strategy, corr) (truncation.jl:330-337)."""
    corr = corr or NoCorrection()
    track = isinstance(corr, (EnergyCorrection, EnergyVarianceCorrection))
    before = expectation_value(v, corr.ket) if track else None
    vbefore = variance(v, corr.ket) if isinstance(corr, EnergyVarianceCorrection) else None
    _apply_(v, strategy)
    if track:
        corr.accumulated_energy += expectation_value(v, corr.ket) - before
        if vbefore is not None:
            corr.accumulated_variance += variance(v, corr.ket) - vbefore
    elif not isinstance(corr, NoCorrection):
        raise NotImplementedError(f"{type(corr).__name__} has no GPU path (no CPU fallback)")
    return v


def _channel(v, kind, prm, qubits):
    m = pack_word(v.N, qubit_mask(v.N, qubits))
    p = np.asarray(prm, dtype=np.float64)
    check(lib.pp_channel(v._h, kind, _ptr(p), _ptr(m)))
    return v


def pauli_channel_(v, pX, pY, pZ, qubits=None):
    """pauli_channel! (channels.jl:203-221)."""
    return _channel(v, 4, [pX, pY, pZ], qubits)


def depolarizing_channel_(v, p, qubits=None):
    """depolarizing_channel! (channels.jl:223-232)."""
    return _channel(v, 0, [p, 0.0, 0.0], qubits)


def dephasing_channel_(v, p, qubits=None):
    """dephasing_channel! (channels.jl:234-243)."""
    return _channel(v, 1, [p, 0.0, 0.0], qubits)


phase_flip_channel_ = dephasing_channel_


def bit_flip_channel_(v, p, qubits=None):
    """bit_flip_channel! (channels.jl:245-254)."""
    return _channel(v, 2, [p, 0.0, 0.0], qubits)


def bit_phase_flip_channel_(v, p, qubits=None):
    """bit_phase_flip_channel! (channels.jl:256-265)."""
    return _channel(v, 3, [p, 0.0, 0.0], qubits)


def depolarizing_channel(v, p, qubits=None):
    return depolarizing_channel_(v.copy(), p, qubits)


def dephasing_channel(v, p, qubits=None):
    return dephasing_channel_(v.copy(), p, qubits)


def bit_flip_channel(v, p, qubits=None):
    return bit_flip_channel_(v.copy(), p, qubits)


def bit_phase_flip_channel(v, p, qubits=None):
    return bit_phase_flip_channel_(v.copy(), p, qubits)


def pauli_channel(v, pX, pY, pZ, qubits=None):
    return pauli_channel_(v.copy(), pX, pY, pZ, qubits)


def depolarizing_p_for_weight_decay(rate, dt):
    """channels.jl:281-282."""
    return 0.75 * (1.0 - math.exp(-rate * dt))


def expectation_value(v, ket):
    """⟨ψ|v|ψ⟩ for a computational-basis ket given as an integer bit mask."""
    k = pack_word(v.N, int(ket))
    out = c_double()
    check(lib.pp_expect_ket(v._h, _ptr(k), byref(out)))
    return out.value


def stochastic_clip_(v, epsilon, rng=None):
    """stochastic_clip!(v, ε; rng) (spv_evolve.jl:35-52): a term with |c| < ε survives
    with probability |c|/ε, promoted to ε·sign(c); rng seeds the device generator."""
    import random as _random
    check(lib.pp_stochastic_clip(v._h, float(epsilon), draw_seed(rng if rng is not None else _random.Random())))
    return v


def variance(v, ket):
    """variance(O, ψ) (statistics.jl:6-22): ⟨ψ|O²|ψ⟩ − ⟨ψ|O|ψ⟩² for a computational-basis
    ket given as an integer bit mask."""
    k = pack_word(v.N, int(ket))
    out = c_double()
    check(lib.pp_variance(v._h, _ptr(k), byref(out)))
    return out.value


# ----------------------------------------------------------------------------- algebra
def mul_(v, a):
    """mul!(v, a) (spv_ops.jl:12-17): v.c *= a."""
    check(lib.pp_scale(v._h, float(a)))
    return v


def scaled(v, a):
    """v * a, a * v, -v (spv_ops.jl:19-30)."""
    return mul_(v.copy(), a)


def norm(v, p=2):
    """norm(v, p) (spv_ops.jl:57-86) for p = 2, 1, inf or any p > 0."""
    out = c_double()
    check(lib.pp_norm(v._h, float(p), byref(out)))
    return out.value


def tr(v):
    """tr(v) (spv_ops.jl:52-55): the identity coefficient times 2^N, with the
    reference's Int64 power (0 for N >= 64)."""
    out = c_double()
    check(lib.pp_trace(v._h, byref(out)))
    return out.value


def sum_(v1, v2):
    """sum!(v1, v2) (spv_ops.jl:182-190): v1 += v2 by an unfiltered merge."""
    check(lib.pp_sum(v1._h, v2._h, 1.0))
    return v1


def add(v1, v2):
    """v1 + v2 (spv_ops.jl:131-165); zero sums are kept."""
    return sum_(v1.copy(), v2)


def sub(v1, v2):
    """v1 - v2 (spv_ops.jl:167)."""
    out = v1.copy()
    check(lib.pp_sum(out._h, v2._h, -1.0))
    return out


def inner_product(v1, v2):
    """inner_product(v1, v2) (spv_ops.jl:378-399): Σ over shared keys of c1·c2."""
    out = c_double()
    check(lib.pp_inner_product(v1._h, v2._h, byref(out)))
    return out.value


def _product_into(out, a, b, kind):
    check(lib.pp_product(out._h, a._h, b._h, kind))
    return out


def product(a, b):
    """a * b (spv_ops.jl:257-284); raises for an imaginary coefficient, as the
    reference's real-typed product does (InexactError)."""
    return _product_into(SparsePauliVector(a.N, 16, 16), a, b, 0)


def anticommutator_(out, a, b):
    """anticommutator!(out, A, B) (spv_ops.jl:460-470): {A, B} into out."""
    return _product_into(out, a, b, 1)


def anticommutator(a, b):
    """anticommutator(A, B) (spv_ops.jl:479-485)."""
    return anticommutator_(SparsePauliVector(a.N, 16, 16), a, b)


def commutator_(out, a, b):
    """commutator!(out, A, B) (spv_ops.jl:446-458): its coefficients are imaginary, so
    it raises for real (Float64) vectors, as the reference does."""
    return _product_into(out, a, b, 2)


def commutator(a, b):
    """commutator(A, B) (spv_ops.jl:472-477)."""
    return commutator_(SparsePauliVector(a.N, 16, 16), a, b)


def check_spv(v):
    """check_spv (type_SparsePauliVector.jl:263-278): raises on violation."""
    ok = c_int32()
    check(lib.pp_check(v._h, byref(ok)))
    if not ok.value:
        raise _lib.PauliPropError("live keys not strictly increasing")
    return True


def power_table(lam, kmax):
    out = np.zeros(kmax + 1, dtype=np.float64)
    check(lib.pp_power_table(float(lam), int(kmax), _ptr(out)))
    return out
