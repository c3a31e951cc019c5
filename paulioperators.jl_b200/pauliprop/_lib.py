"""ctypes binding of libpauliprop.so (include/pauliprop.h).

The library is built in-tree (paulioperators.jl_b200/lib/libpauliprop.so by
``make -C paulioperators.jl_b200``).  There is no CPU fallback: if the library
is missing, importing this module raises, and on a machine without a CUDA
device every compute entry point returns PP_DEVICE_ERROR, which is raised as
``DeviceError``.
"""
import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int32, c_int64, c_uint8, c_uint64,
                    c_void_p)

from .errors import ArgumentError, DeviceError, DimensionMismatch, PauliPropError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PAULIPROP_LIB") or os.path.join(os.path.dirname(_HERE), "lib", "libpauliprop.so")

PP_OK = 0
PP_ARGUMENT_ERROR = 1
PP_DIMENSION_MISMATCH = 2
PP_ERROR_EXCEPTION = 3
PP_OUT_OF_MEMORY = 4
PP_DEVICE_ERROR = 5
PP_TIMEOUT = 6
PP_NOT_IMPLEMENTED = 7


class PPFilter(Structure):
    """pp_filter == the reference's isbits MergeFilter (spv_kernels.jl:33-42)."""
    _fields_ = [("wmax", c_int64), ("xwmax", c_int64), ("mwmax", c_int64),
                ("thresh", c_double), ("alpha_w", c_double), ("dthresh_w", c_double),
                ("alpha_xw", c_double), ("dthresh_xw", c_double)]


class PPCounters(Structure):
    _fields_ = [("nwin", c_int64),
                ("terms_created", POINTER(c_int64)), ("merge_in", POINTER(c_int64)),
                ("merge_out", POINTER(c_int64)), ("early_merges", POINTER(c_int64)),
                ("t_rotate", POINTER(c_double)), ("t_merge", POINTER(c_double))]


class PPEvolveOpts(Structure):
    _fields_ = [("window", c_int64),
                ("strict", POINTER(PPFilter)), ("local", POINTER(PPFilter)),
                ("strict_kind", c_int32), ("corr_kind", c_int32),
                ("adapt_max_terms", c_int64), ("adapt_min_thresh", c_double),
                ("ket", c_void_p), ("corr_energy", POINTER(c_double)),
                ("counters", POINTER(PPCounters)),
                ("chan_kind", c_int32), ("pad", c_int32),
                ("chan_prm", c_double * 3), ("chan_mask", c_void_p),
                ("expect_out", POINTER(c_double)),
                ("chan_every", c_int64), ("stats_out", POINTER(c_double)),
                ("profile", c_int32), ("pad2", c_int32), ("corr_variance", POINTER(c_double)),
                ("seed", c_uint64)]


class PPBatch(Structure):
    _fields_ = [("ninst", c_int64), ("nq", c_int32), ("ncol", c_int32),
                ("acol", c_void_p), ("cosv", c_void_p), ("sinv", c_void_p), ("rot_end", c_void_p),
                ("keep_finished", c_int32), ("pad", c_int32),
                ("expect_out", c_void_p), ("t_done", c_void_p), ("n_final", c_void_p)]


class PPFeatureCtx(Structure):
    _fields_ = [("nq", c_int32), ("pad", c_int32), ("nbr", c_uint64 * 64), ("light_cone", c_uint64),
                ("boundary", c_uint64), ("row", c_uint8 * 64), ("col", c_uint8 * 64),
                ("layer_frac", c_float), ("remaining_frac", c_float), ("theta_j", c_float), ("theta_h", c_float)]


class PPDropSample(Structure):
    _fields_ = [("cap", c_int64), ("seed", c_uint64), ("z", c_void_p), ("x", c_void_p), ("c", c_void_p),
                ("n", c_int64), ("n_dropped", c_int64)]


class PPTuning(Structure):
    _fields_ = [("bucket_cap", c_int32), ("items_per_thread", c_int32), ("load_div", c_int32), ("chunk", c_int32)]


PP_MLP_NPARAM = 5313
PP_STATS_LEN = 16
STAT = {"terms_in": 0, "created": 1, "merge_in": 2, "merge_out": 3, "peak": 4, "early": 5,
        "t_rotate": 6, "t_merge": 7, "launches": 8, "t_partition": 9, "bucket_rot": 10, "bucket_bytes": 11}


# Every symbol include/pauliprop.h declares, with its ctypes signature.
SIGNATURES = {
    "pp_create": (c_int32, [c_int32, c_int64, c_int64, POINTER(c_void_p)]),
    "pp_destroy": (c_int32, [c_void_p]),
    "pp_upload": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32]),
    "pp_download": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, POINTER(c_int64)]),
    "pp_length": (c_int32, [c_void_p, POINTER(c_int64)]),
    "pp_copy": (c_int32, [c_void_p, POINTER(c_void_p)]),
    "pp_evolve1": (c_int32, [c_void_p, c_void_p, c_void_p, c_double, c_double]),
    "pp_evolve": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, POINTER(PPEvolveOpts)]),
    "pp_compact": (c_int32, [c_void_p, POINTER(PPFilter)]),
    "pp_evolve_batch": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64, POINTER(PPBatch),
                                  POINTER(PPEvolveOpts)]),
    "pp_compact_static": (c_int32, [c_int32, c_void_p, c_void_p, c_void_p, c_int64, POINTER(PPFilter),
                                    c_void_p, c_void_p, c_void_p, POINTER(c_int64), c_void_p]),
    "pp_adaptive": (c_int32, [c_void_p, c_int64, c_double]),
    "pp_channel": (c_int32, [c_void_p, c_int32, c_void_p, c_void_p]),
    "pp_expect_ket": (c_int32, [c_void_p, c_void_p, POINTER(c_double)]),
    "pp_variance": (c_int32, [c_void_p, c_void_p, POINTER(c_double)]),
    "pp_stochastic_clip": (c_int32, [c_void_p, c_double, c_uint64]),
    "pp_stochastic_sample": (c_int32, [c_void_p, c_int64, c_uint64]),
    "pp_check": (c_int32, [c_void_p, POINTER(c_int32)]),
    "pp_stream": (c_int32, [c_void_p, POINTER(c_void_p)]),
    "pp_device_bytes": (c_int32, [c_void_p, POINTER(c_int64)]),
    "pp_power_table": (c_int32, [c_double, c_int32, c_void_p]),
    "pp_mlp_create": (c_int32, [POINTER(c_void_p)]),
    "pp_mlp_destroy": (c_int32, [c_void_p]),
    "pp_mlp_set_params": (c_int32, [c_void_p, c_void_p]),
    "pp_mlp_get_params": (c_int32, [c_void_p, c_void_p]),
    "pp_mlp_forward": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p]),
    "pp_mlp_grad": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, POINTER(c_float)]),
    "pp_mlp_load_data": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64]),
    "pp_mlp_train": (c_int32, [c_void_p, c_int64, c_int64, c_float, c_uint64, c_void_p]),
    "pp_features": (c_int32, [c_void_p, POINTER(PPFeatureCtx), c_void_p, c_int64, POINTER(c_int64)]),
    "pp_learned_truncate": (c_int32, [c_void_p, c_void_p, POINTER(PPFeatureCtx), c_int64, POINTER(c_float),
                                      POINTER(PPDropSample)]),
    "pp_sample_terms": (c_int32, [c_void_p, c_int32, c_double, c_double, c_int64, c_uint64, c_void_p, c_void_p,
                                  c_void_p, c_int64, POINTER(c_int64)]),
    "pp_scale": (c_int32, [c_void_p, c_double]),
    "pp_norm": (c_int32, [c_void_p, c_double, POINTER(c_double)]),
    "pp_trace": (c_int32, [c_void_p, POINTER(c_double)]),
    "pp_sum": (c_int32, [c_void_p, c_void_p, c_double]),
    "pp_inner_product": (c_int32, [c_void_p, c_void_p, POINTER(c_double)]),
    "pp_product": (c_int32, [c_void_p, c_void_p, c_void_p, c_int32]),
    "pp_last_error": (c_char_p, []),
    "pp_set_tuning": (c_int32, [c_void_p, POINTER(PPTuning)]),
    "pp_get_tuning": (c_int32, [c_void_p, POINTER(PPTuning)]),
    "pp_device_info": (c_int32, [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]),
    "pp_debug_fail_alloc": (c_int32, [c_int64]),
    "pp_debug_lookback_timeout": (c_int32, [c_int64]),
    "pp_debug_bucket_limit": (c_int32, [c_int64]),
    "pp_shard_owner": (c_int32, [c_int32, c_void_p, c_void_p, c_int64, c_int32, c_void_p]),
    "pp_shard_begin": (c_int32, [c_void_p, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                 POINTER(PPEvolveOpts), c_int32, c_void_p]),
    "pp_shard_send": (c_int32, [c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p, c_int64, c_void_p,
                                c_void_p]),
    "pp_shard_recv": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64]),
    "pp_shard_rotate": (c_int32, [c_void_p, c_int64, c_int32, c_void_p]),
    "pp_shard_regrid": (c_int32, [c_void_p, c_int32, c_void_p]),
    "pp_shard_end": (c_int32, [c_void_p, c_void_p, c_void_p]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libpauliprop.so not found at {LIB_PATH}; build it with "
            "`make -C paulioperators.jl_b200` (there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status):
    """Raise the Python analogue of the reference's exception for a pp_status."""
    if status == PP_OK:
        return
    msg = (lib.pp_last_error() or b"").decode(errors="replace")
    if status == PP_ARGUMENT_ERROR:
        raise ArgumentError(msg)
    if status == PP_DIMENSION_MISMATCH:
        raise DimensionMismatch(msg)
    if status == PP_ERROR_EXCEPTION:
        raise PauliPropError(msg)
    if status == PP_OUT_OF_MEMORY:
        raise MemoryError(msg)
    if status == PP_TIMEOUT:
        raise TimeoutError(msg)
    if status == PP_NOT_IMPLEMENTED:
        raise NotImplementedError(msg)
    raise DeviceError(msg)
