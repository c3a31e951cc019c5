"""The C-ABI library loads, exports every symbol include/pauliprop.h declares, and
its host-only helpers work; compute entry points need a GPU (not called here)."""
import ctypes
import os
import re

import numpy as np
import pytest

import orc
import pauliprop as pp
from conftest import ROOT, has_gpu
from pauliprop import _lib


def header_symbols():
    src = open(os.path.join(ROOT, "include", "pauliprop.h")).read()
    return sorted(set(re.findall(r"\b(pp_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 16
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES)


def test_last_error_and_argument_checks_without_device():
    out = ctypes.c_void_p()
    assert _lib.lib.pp_create(200, 16, 16, ctypes.byref(out)) == _lib.PP_ERROR_EXCEPTION
    assert b"128" in _lib.lib.pp_last_error()
    assert _lib.lib.pp_power_table(0.5, -1, None) == _lib.PP_ARGUMENT_ERROR


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_create_without_gpu_fails_loudly():
    with pytest.raises(pp.DeviceError):
        pp.SparsePauliVector(8)


def test_power_table_matches_oracle_bitwise():
    for lam in (1 - 4 * 1e-3 / 3, 1 - 2 * 5e-4, 0.37, 1 - 2 * (0.1 + 0.15)):
        t = pp.power_table(lam, 128)
        for k in range(129):
            assert t[k] == orc.jl_pow(lam, k)


def test_struct_layouts():
    assert ctypes.sizeof(_lib.PPFilter) == 64
    assert ctypes.sizeof(_lib.PPEvolveOpts) == 144
    assert ctypes.sizeof(_lib.PPCounters) == 56
