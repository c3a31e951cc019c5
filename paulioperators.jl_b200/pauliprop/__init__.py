"""pauliprop: B200-native SparsePauliVector Pauli propagation.

Python host mirror of PauliOperators.jl's SparsePauliVector propagation API
over libpauliprop.so (C ABI in include/pauliprop.h).
"""
from ._lib import (ArgumentError, DeviceError, DimensionMismatch, PauliPropError, LIB_PATH)
from .paulis import (PauliBasis, PauliSum, majorana_weight, nwords, pack_keys, pack_word,
                     qubit_mask, unpack_keys, weight, x_weight)
from .truncation import (NOFILTER, AdaptiveTruncation, CoeffTruncation, CompositeTruncation,
                         CorrectionAccumulator, EnergyCorrection, EnergyVarianceCorrection,
                         MajoranaWeightTruncation, MergeFilter, NoCorrection, NoTruncation,
                         StochasticCoeffTruncation, StochasticSamplingTruncation,
                         TruncationStrategy, WeightDampedTruncation, WeightTruncation,
                         XWeightDampedTruncation, XWeightTruncation, combine_filters,
                         compile_filter, is_compilable)
from .spv import (SparsePauliVector, WindowCounters, add, anticommutator, anticommutator_, commutator,
                  commutator_, inner_product, mul_, norm, product, scaled, sub, sum_, tr, bit_flip_channel, bit_flip_channel_,
                  bit_phase_flip_channel, bit_phase_flip_channel_, check_spv, clip_,
                  coeff_clip_, dephasing_channel, dephasing_channel_, depolarizing_channel,
                  depolarizing_channel_, depolarizing_p_for_weight_decay, evolve, evolve_,
                  expectation_value, majorana_weight_clip_, pauli_channel, pauli_channel_,
                  phase_flip_channel_, power_table, truncate_, weight_clip_,
                  weight_damped_clip_, stochastic_clip_, variance, x_weight_clip_,
                  x_weight_damped_clip_)
from .batch import BatchResult, evolve_batch, split_instances, tagged_terms
from .learned import MLP, features, lattice_feature_ctx, learned_truncate_
from . import circuits

__all__ = [n for n in dir() if not n.startswith("_")]
