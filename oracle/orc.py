"""CPU ORACLE wrapper — test infrastructure only.

ctypes binding of oracle/_build/liborc.so, the plain-C restatement of the
reference SparsePauliVector path (see spv_oracle.h for what pins it).  Used by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs as the
checker; the product library never loads it.
"""
import ctypes
import math
import os
import subprocess
from ctypes import POINTER, Structure, c_char_p, c_double, c_int, c_int32, c_int64, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liborc.so")
INT64_MAX = 2**63 - 1
NOFILTER = (INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0)


class OrcFilter(Structure):
    _fields_ = [("wmax", c_int64), ("xwmax", c_int64), ("mwmax", c_int64),
                ("thresh", c_double), ("alpha_w", c_double), ("dthresh_w", c_double),
                ("alpha_xw", c_double), ("dthresh_xw", c_double)]


class OrcParams(Structure):
    _fields_ = [("window", c_int64), ("strict", OrcFilter), ("strict_compiled", c_int32),
                ("corr_kind", c_int32), ("adapt_max_terms", c_int64), ("adapt_min_thresh", c_double),
                ("local", OrcFilter), ("ket", c_uint64 * 2), ("corr_energy", c_double),
                ("nwin", c_int64), ("terms_created", POINTER(c_int64)), ("merge_in", POINTER(c_int64)),
                ("merge_out", POINTER(c_int64)), ("early_merges", POINTER(c_int64))]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    sig = {
        "orc_create": (c_void_p, [c_int, c_int64, c_int64]),
        "orc_destroy": (None, [c_void_p]),
        "orc_nwords": (c_int, [c_void_p]),
        "orc_len": (c_int64, [c_void_p]),
        "orc_live_cap": (c_int64, [c_void_p]),
        "orc_append_cap": (c_int64, [c_void_p]),
        "orc_upload": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64]),
        "orc_download": (c_int64, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64]),
        "orc_copy": (c_void_p, [c_void_p]),
        "orc_evolve1": (c_int, [c_void_p, c_void_p, c_void_p, c_double, c_double]),
        "orc_evolve": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, POINTER(OrcParams)]),
        "orc_compact": (c_int, [c_void_p, POINTER(OrcFilter)]),
        "orc_adaptive": (c_int, [c_void_p, c_int64, c_double]),
        "orc_channel": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
        "orc_expect": (c_double, [c_void_p, c_void_p]),
        "orc_expect_neumaier": (c_double, [c_void_p, c_void_p]),
        "orc_check": (c_int, [c_void_p]),
        "orc_jl_pow": (c_double, [c_double, c_int64]),
        "orc_last_error": (c_char_p, []),
    }
    for k, (r, a) in sig.items():
        f = getattr(lib, k)
        f.restype = r
        f.argtypes = a
    return lib


lib = _load()


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


def _chk(code):
    if code != 0:
        raise OracleError(code, (lib.orc_last_error() or b"").decode())


def _p(a):
    return a.ctypes.data_as(c_void_p) if a is not None else None


def nwords(N):
    return 1 if N <= 64 else 2


def word(N, v):
    m = (1 << 64) - 1
    return np.array([(int(v) >> (64 * w)) & m for w in range(nwords(N))], dtype=np.uint64)


def words(N, vals):
    nw = nwords(N)
    m = (1 << 64) - 1
    a = np.zeros((len(vals), nw), dtype=np.uint64)
    for i, v in enumerate(vals):
        for w in range(nw):
            a[i, w] = (int(v) >> (64 * w)) & m
    return a


class OracleSPV:
    """The reference SparsePauliVector, restated in C (single-threaded)."""

    def __init__(self, N, live_cap=16, append_cap=None, _h=None):
        self.N = N
        self.nw = nwords(N)
        if _h is None:
            _h = lib.orc_create(N, max(1, live_cap), max(1, append_cap if append_cap is not None else live_cap))
            if not _h:
                raise OracleError(3, (lib.orc_last_error() or b"").decode())
        self._h = _h

    @classmethod
    def from_terms(cls, N, terms, capacity_factor=2.0, append_factor=1.0, min_capacity=16):
        """SparsePauliVector(O::PauliSum; ...) sizing (type_SparsePauliVector.jl:173-176)."""
        live_cap = max(min_capacity, math.ceil(capacity_factor * max(len(terms), 1)))
        append_cap = max(min_capacity, math.ceil(append_factor * live_cap))
        v = cls(N, live_cap, append_cap)
        v.upload([t[0] for t in terms], [t[1] for t in terms], [t[2] for t in terms])
        return v

    def upload(self, zs, xs, cs):
        z = zs if isinstance(zs, np.ndarray) and zs.dtype == np.uint64 else words(self.N, zs)
        x = xs if isinstance(xs, np.ndarray) and xs.dtype == np.uint64 else words(self.N, xs)
        c = np.ascontiguousarray(cs, dtype=np.float64)
        _chk(lib.orc_upload(self._h, _p(np.ascontiguousarray(z)), _p(np.ascontiguousarray(x)), _p(c), len(c)))

    def arrays(self):
        n = len(self)
        z = np.zeros((n, self.nw), dtype=np.uint64)
        x = np.zeros((n, self.nw), dtype=np.uint64)
        c = np.zeros(n, dtype=np.float64)
        lib.orc_download(self._h, _p(z), _p(x), _p(c), n)
        return z, x, c

    def terms(self):
        z, x, c = self.arrays()
        out = {}
        for i in range(len(c)):
            kz = sum(int(z[i, w]) << (64 * w) for w in range(self.nw))
            kx = sum(int(x[i, w]) << (64 * w) for w in range(self.nw))
            out[(kz, kx)] = float(c[i])
        return out

    def __len__(self):
        return lib.orc_len(self._h)

    @property
    def append_cap(self):
        return lib.orc_append_cap(self._h)

    def copy(self):
        return OracleSPV(self.N, _h=lib.orc_copy(self._h))

    def evolve1(self, gz, gx, theta):
        _chk(lib.orc_evolve1(self._h, _p(word(self.N, gz)), _p(word(self.N, gx)), math.cos(theta), math.sin(theta)))

    def evolve(self, gens, angles, window=1, strict=NOFILTER, local=NOFILTER, adaptive=None,
               energy_ket=None, energy0=0.0, nwin=0):
        """Sequence evolve!; gens: list of (z, x) ints; returns (accumulated_energy, counters)."""
        L = len(gens)
        gz = words(self.N, [g[0] for g in gens])
        gx = words(self.N, [g[1] for g in gens])
        cs = np.array([math.cos(a) for a in angles], dtype=np.float64)
        ss = np.array([math.sin(a) for a in angles], dtype=np.float64)
        p = OrcParams()
        p.window = window
        p.strict = OrcFilter(*strict)
        p.strict_compiled = 0 if adaptive else 1
        if adaptive:
            p.adapt_max_terms, p.adapt_min_thresh = adaptive
        p.local = OrcFilter(*local)
        p.corr_kind = 1 if energy_ket is not None else 0
        if energy_ket is not None:
            m = (1 << 64) - 1
            p.ket[0] = int(energy_ket) & m
            p.ket[1] = (int(energy_ket) >> 64) & m
        p.corr_energy = energy0
        ctr = None
        if nwin:
            ctr = [np.zeros(nwin, dtype=np.int64) for _ in range(4)]
            P64 = POINTER(c_int64)
            p.nwin = nwin
            p.terms_created, p.merge_in, p.merge_out, p.early_merges = [a.ctypes.data_as(P64) for a in ctr]
        _chk(lib.orc_evolve(self._h, _p(gz), _p(gx), _p(cs), _p(ss), L, ctypes.byref(p)))
        return p.corr_energy, ctr

    def compact(self, f):
        _chk(lib.orc_compact(self._h, ctypes.byref(OrcFilter(*f))))

    def adaptive(self, max_terms, min_thresh):
        _chk(lib.orc_adaptive(self._h, max_terms, min_thresh))

    def channel(self, kind, prm, mask=None):
        pr = np.asarray(list(prm) + [0.0] * (3 - len(prm)), dtype=np.float64)
        m = word(self.N, mask) if mask is not None else None
        _chk(lib.orc_channel(self._h, kind, _p(pr), _p(m)))

    def expect(self, ket=0):
        return lib.orc_expect(self._h, _p(word(self.N, ket)))

    def expect_neumaier(self, ket=0):
        return lib.orc_expect_neumaier(self._h, _p(word(self.N, ket)))

    def check(self):
        return bool(lib.orc_check(self._h))

    def __del__(self):
        if getattr(self, "_h", None):
            lib.orc_destroy(self._h)
            self._h = None


def jl_pow(x, n):
    return lib.orc_jl_pow(x, n)
