"""Truncation strategies and correction accumulators (src/truncation.jl) and
their compilation into the per-term MergeFilter predicate
(_compile_filter / _combine_filters / _is_compilable, spv_kernels.jl:81-125).
"""
import random
from collections import namedtuple

from .paulis import INT64_MAX

MergeFilter = namedtuple(
    "MergeFilter", "wmax xwmax mwmax thresh alpha_w dthresh_w alpha_xw dthresh_xw")

# NOFILTER (spv_kernels.jl:44-45): keeps exact zeros (thresh = -1).
NOFILTER = MergeFilter(INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0)


class TruncationStrategy:
    """Abstract supertype (truncation.jl:14)."""


class NoTruncation(TruncationStrategy):
    """Identity truncation (truncation.jl:37)."""


class CoeffTruncation(TruncationStrategy):
    """Drop |c| <= thresh (truncation.jl:44-47)."""

    def __init__(self, thresh=1e-6):
        self.thresh = float(thresh)


class WeightTruncation(TruncationStrategy):
    """Drop Pauli weight > max_weight (truncation.jl:54-56)."""

    def __init__(self, max_weight):
        self.max_weight = int(max_weight)


class XWeightTruncation(TruncationStrategy):
    """Drop X-weight > max_weight (truncation.jl:63-65)."""

    def __init__(self, max_weight):
        self.max_weight = int(max_weight)


class MajoranaWeightTruncation(TruncationStrategy):
    """Drop Majorana weight > max_weight (truncation.jl:72-74)."""

    def __init__(self, max_weight):
        self.max_weight = int(max_weight)


class WeightDampedTruncation(TruncationStrategy):
    """Drop |c| exp(-alpha w) <= thresh (truncation.jl:84-88)."""

    def __init__(self, alpha, thresh=1e-6):
        self.alpha = float(alpha)
        self.thresh = float(thresh)


class XWeightDampedTruncation(TruncationStrategy):
    """Drop |c| exp(-alpha x_weight) <= thresh (truncation.jl:98-102)."""

    def __init__(self, alpha, thresh=1e-6):
        self.alpha = float(alpha)
        self.thresh = float(thresh)


def draw_seed(rng):
    """A 64-bit seed for the device generator from a random.Random, a numpy
    Generator or an integer (each use of a strategy draws a fresh one, so repeated
    truncations are independent, as with the reference's advancing RNG)."""
    if isinstance(rng, int):
        return rng & ((1 << 64) - 1)
    if hasattr(rng, "getrandbits"):
        return rng.getrandbits(64)
    return int(rng.integers(0, 1 << 63)) << 1 | int(rng.integers(0, 2))


class StochasticCoeffTruncation(TruncationStrategy):
    """Russian roulette (truncation.jl:105-117); device random numbers seeded from rng."""

    def __init__(self, epsilon, rng=None):
        self.epsilon = float(epsilon)
        self.rng = rng if rng is not None else random.Random()


class StochasticSamplingTruncation(TruncationStrategy):
    """|c|^2 importance sampling (truncation.jl:119-129); device random numbers seeded from rng."""

    def __init__(self, n_keep, rng=None):
        self.n_keep = int(n_keep)
        self.rng = rng if rng is not None else random.Random()


class AdaptiveTruncation(TruncationStrategy):
    """Top-max_terms threshold, else min_thresh (truncation.jl:137-141)."""

    def __init__(self, max_terms=10000, min_thresh=1e-12):
        self.max_terms = int(max_terms)
        self.min_thresh = float(min_thresh)


class CompositeTruncation(TruncationStrategy):
    """Sequential composition (truncation.jl:155-159)."""

    def __init__(self, *strategies):
        if len(strategies) == 1 and isinstance(strategies[0], (list, tuple)):
            strategies = tuple(strategies[0])
        self.strategies = tuple(strategies)


class CorrectionAccumulator:
    """Abstract supertype (truncation.jl:25)."""


class NoCorrection(CorrectionAccumulator):
    """Track nothing (truncation.jl:255)."""


class EnergyCorrection(CorrectionAccumulator):
    """Accumulated change of <ψ|O|ψ> through truncation (truncation.jl:262-266)."""

    def __init__(self, ket):
        self.ket = int(ket)
        self.accumulated_energy = 0.0


class EnergyVarianceCorrection(CorrectionAccumulator):
    """Energy and variance tracking (truncation.jl:269-278)."""

    def __init__(self, ket):
        self.ket = int(ket)
        self.accumulated_energy = 0.0
        self.accumulated_variance = 0.0


_SIMPLE = (NoTruncation, CoeffTruncation, WeightTruncation, XWeightTruncation,
           MajoranaWeightTruncation, WeightDampedTruncation, XWeightDampedTruncation)


def is_compilable(s):
    """_is_compilable (spv_kernels.jl:116-125)."""
    if isinstance(s, CompositeTruncation):
        if not all(is_compilable(x) for x in s.strategies):
            return False
        if sum(isinstance(x, WeightDampedTruncation) for x in s.strategies) > 1:
            return False
        if sum(isinstance(x, XWeightDampedTruncation) for x in s.strategies) > 1:
            return False
        return True
    return isinstance(s, _SIMPLE)


def combine_filters(f1, f2):
    """_combine_filters (spv_kernels.jl:98-108)."""
    if f1.dthresh_w >= 0 and f2.dthresh_w >= 0:
        raise RuntimeError("cannot combine two weight-damped truncations in one composite")
    if f1.dthresh_xw >= 0 and f2.dthresh_xw >= 0:
        raise RuntimeError("cannot combine two x-weight-damped truncations in one composite")
    dw = f1 if f1.dthresh_w >= 0 else f2
    dxw = f1 if f1.dthresh_xw >= 0 else f2
    return MergeFilter(min(f1.wmax, f2.wmax), min(f1.xwmax, f2.xwmax),
                       min(f1.mwmax, f2.mwmax), max(f1.thresh, f2.thresh),
                       dw.alpha_w, dw.dthresh_w, dxw.alpha_xw, dxw.dthresh_xw)


def compile_filter(s):
    """_compile_filter (spv_kernels.jl:81-111)."""
    if isinstance(s, NoTruncation):
        return NOFILTER
    if isinstance(s, CoeffTruncation):
        return MergeFilter(INT64_MAX, INT64_MAX, INT64_MAX, s.thresh, 0.0, -1.0, 0.0, -1.0)
    if isinstance(s, WeightTruncation):
        return MergeFilter(s.max_weight, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0)
    if isinstance(s, XWeightTruncation):
        return MergeFilter(INT64_MAX, s.max_weight, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0)
    if isinstance(s, MajoranaWeightTruncation):
        return MergeFilter(INT64_MAX, INT64_MAX, s.max_weight, -1.0, 0.0, -1.0, 0.0, -1.0)
    if isinstance(s, WeightDampedTruncation):
        return MergeFilter(INT64_MAX, INT64_MAX, INT64_MAX, -1.0, s.alpha, s.thresh, 0.0, -1.0)
    if isinstance(s, XWeightDampedTruncation):
        return MergeFilter(INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, s.alpha, s.thresh)
    if isinstance(s, CompositeTruncation):
        f = NOFILTER
        for x in s.strategies:
            f = combine_filters(f, compile_filter(x))
        return f
    raise RuntimeError(f"{type(s).__name__} cannot be compiled to a MergeFilter "
                       "(internal misuse: check is_compilable before compiling)")
