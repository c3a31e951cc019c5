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
    """The ctypes mirrors have the sizes and field offsets of include/pauliprop.h's
    structs, as gcc lays them out."""
    import os
    import subprocess
    import tempfile
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    structs = {"pp_filter": _lib.PPFilter, "pp_evolve_opts": _lib.PPEvolveOpts, "pp_counters": _lib.PPCounters,
               "pp_batch": _lib.PPBatch, "pp_feature_ctx": _lib.PPFeatureCtx, "pp_drop_sample": _lib.PPDropSample,
               "pp_tuning": _lib.PPTuning}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pauliprop.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        with open(src, "w") as f:
            f.write("\n".join(lines))
        subprocess.run(["gcc", "-I", os.path.join(root, "include"), src, "-o", exe], check=True)
        out = dict(l.rsplit(" ", 1) for l in subprocess.run([exe], check=True, capture_output=True,
                                                            text=True).stdout.split("\n") if l)
    for cname, py in structs.items():
        assert int(out[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)
