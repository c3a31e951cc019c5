"""pauliprop: B200-native SparsePauliVector Pauli propagation.

Python host mirror of PauliOperators.jl's SparsePauliVector propagation API
over libpauliprop.so (C ABI in include/pauliprop.h).

The strategy types, Pauli strings and circuit builders are plain host code and
import without the library.  Every device-backed name (SparsePauliVector,
evolve_, the channels, the algebra, batched instances, learned truncation) is
bound on first use, which loads libpauliprop.so: without the library that
first use raises ImportError (there is no CPU fallback).
"""
import importlib

from .errors import ArgumentError, DeviceError, DimensionMismatch, PauliPropError
from .paulis import (PauliBasis, PauliSum, majorana_weight, nwords, pack_keys, pack_word,
                     qubit_mask, unpack_keys, weight, x_weight)
from .truncation import (NOFILTER, AdaptiveTruncation, CoeffTruncation, CompositeTruncation,
                         CorrectionAccumulator, EnergyCorrection, EnergyVarianceCorrection,
                         MajoranaWeightTruncation, MergeFilter, NoCorrection, NoTruncation,
                         StochasticCoeffTruncation, StochasticSamplingTruncation,
                         TruncationStrategy, WeightDampedTruncation, WeightTruncation,
                         XWeightDampedTruncation, XWeightTruncation, combine_filters,
                         compile_filter, is_compilable)
from . import circuits

_DEVICE_NAMES = {
    "spv": ("SparsePauliVector", "WindowCounters", "add", "anticommutator", "anticommutator_", "commutator",
            "commutator_", "inner_product", "mul_", "norm", "product", "scaled", "sub", "sum_", "tr",
            "bit_flip_channel", "bit_flip_channel_", "bit_phase_flip_channel", "bit_phase_flip_channel_",
            "check_spv", "clip_", "coeff_clip_", "dephasing_channel", "dephasing_channel_",
            "depolarizing_channel", "depolarizing_channel_", "depolarizing_p_for_weight_decay", "evolve",
            "evolve_", "expectation_value", "majorana_weight_clip_", "pauli_channel", "pauli_channel_",
            "phase_flip_channel_", "power_table", "truncate_", "weight_clip_", "weight_damped_clip_",
            "stochastic_clip_", "variance", "x_weight_clip_", "x_weight_damped_clip_"),
    "batch": ("BatchResult", "evolve_batch", "split_instances", "tagged_terms"),
    "learned": ("MLP", "features", "lattice_feature_ctx", "learned_truncate_"),
    "_lib": ("LIB_PATH",),
}
_LAZY = {name: mod for mod, names in _DEVICE_NAMES.items() for name in names}
_LAZY_MODULES = ("spv", "batch", "learned", "_lib", "tune")


def __getattr__(name):
    """Binds a device-backed name (or submodule) on first use; this loads libpauliprop.so."""
    if name in _LAZY_MODULES:
        return importlib.import_module("." + name, __name__)
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(f"module 'pauliprop' has no attribute {name!r}")
    value = getattr(importlib.import_module("." + mod, __name__), name)
    globals()[name] = value
    return value


def __dir__():
    return sorted(set(globals()) | set(_LAZY))


__all__ = sorted(n for n in set(globals()) | set(_LAZY) if not n.startswith("_") and n != "importlib")
