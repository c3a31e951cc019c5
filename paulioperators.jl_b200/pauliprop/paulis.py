"""Host-side Pauli strings and packing, mirroring PauliOperators.jl conventions.

PauliBasis{N}(z, x) (src/type_PauliBasis.jl:15-21): qubit q (1-based) is bit
q-1 of z and x; X sets x, Z sets z, Y sets both.  The packed word type follows
_word_type (src/type_SparsePauliVector.jl:23-26): one uint64 per term for
N <= 64, two (low, high) for N <= 128.
"""
import numpy as np

from .errors import PauliPropError

INT64_MAX = 2**63 - 1


def nwords(N):
    """Number of 64-bit words of the packed word type (_word_type)."""
    if N <= 64:
        return 1
    if N <= 128:
        return 2
    raise PauliPropError("N > 128 requires a multi-word type (add BitIntegers.jl and extend _word_type)")


class PauliBasis:
    """A Hermitian Pauli string P_1 ⊗ ... ⊗ P_N as (z, x) bit masks."""
    __slots__ = ("N", "z", "x")

    def __init__(self, N, z, x):
        self.N = int(N)
        self.z = int(z)
        self.x = int(x)

    @classmethod
    def from_string(cls, s):
        """PauliBasis(str) (type_PauliBasis.jl:38-64): character i sets bit i-1."""
        z = x = 0
        for i, ch in enumerate(s):
            if ch not in "IXYZ":
                raise ValueError(f"Bad string: {s}")
            if ch in "XY":
                x |= 1 << i
            if ch in "ZY":
                z |= 1 << i
        return cls(len(s), z, x)

    @classmethod
    def from_sites(cls, N, X=(), Y=(), Z=()):
        """Pauli(N; X=[...], Y=[...], Z=[...]) with 1-based qubit indices."""
        z = x = 0
        for q in X:
            x |= 1 << (q - 1)
        for q in Y:
            x |= 1 << (q - 1)
            z |= 1 << (q - 1)
        for q in Z:
            z |= 1 << (q - 1)
        return cls(N, z, x)

    def __str__(self):
        out = []
        for i in range(self.N):
            zb, xb = (self.z >> i) & 1, (self.x >> i) & 1
            out.append("Y" if zb and xb else "X" if xb else "Z" if zb else "I")
        return "".join(out)

    __repr__ = __str__

    def key(self):
        return (self.z, self.x)

    def __eq__(self, o):
        return isinstance(o, PauliBasis) and (self.N, self.z, self.x) == (o.N, o.z, o.x)

    def __hash__(self):
        return hash((self.N, self.z, self.x))


def weight(z, x):
    """weight (clip.jl:6-8): number of non-identity factors."""
    return bin(z | x).count("1")


def x_weight(z, x):
    """x_weight (clip.jl:53-55)."""
    return bin(x).count("1")


def majorana_weight(N, z, x):
    """majorana_weight (clip.jl:88-117) on the 128-bit reference representation."""
    M = (1 << 128) - 1
    zbits = z & ~x & M
    S = x & M
    for s in (1, 2, 4, 8, 16, 32, 64):
        S ^= S >> s
    ctrl = ~(S ^ x) & M
    return (bin(x).count("1") + 2 * bin(zbits & ctrl).count("1")
            + 2 * bin(~(z | x) & ~ctrl & M).count("1"))


class PauliSum(dict):
    """Dict-backed PauliSum{N,T} (type_PauliSum.jl:8): {(z, x): coefficient}."""

    def __init__(self, N, items=None):
        super().__init__()
        self.N = int(N)
        if items:
            for k, v in dict(items).items():
                self[k] = v

    def __setitem__(self, k, v):
        if isinstance(k, PauliBasis):
            k = k.key()
        elif isinstance(k, str):
            k = PauliBasis.from_string(k).key()
        super().__setitem__((int(k[0]), int(k[1])), v)

    def __getitem__(self, k):
        if isinstance(k, PauliBasis):
            k = k.key()
        elif isinstance(k, str):
            k = PauliBasis.from_string(k).key()
        return super().__getitem__(k)

    def copy(self):
        return PauliSum(self.N, dict(self))


def pack_keys(N, keys):
    """Pack integer (z, x) pairs into word arrays of the reference word type."""
    nw = nwords(N)
    n = len(keys)
    z = np.zeros((n, nw), dtype=np.uint64)
    x = np.zeros((n, nw), dtype=np.uint64)
    m = (1 << 64) - 1
    for i, (kz, kx) in enumerate(keys):
        for w in range(nw):
            z[i, w] = (kz >> (64 * w)) & m
            x[i, w] = (kx >> (64 * w)) & m
    return z, x


def pack_word(N, v):
    """One packed word (array of nwords uint64) for a bit mask / ket."""
    nw = nwords(N)
    m = (1 << 64) - 1
    return np.array([(int(v) >> (64 * w)) & m for w in range(nw)], dtype=np.uint64)


def unpack_keys(z, x):
    """Inverse of pack_keys: list of (z, x) Python ints."""
    z = np.asarray(z, dtype=np.uint64).reshape(len(z), -1)
    x = np.asarray(x, dtype=np.uint64).reshape(len(x), -1)
    nw = z.shape[1]
    out = []
    for i in range(z.shape[0]):
        kz = kx = 0
        for w in range(nw):
            kz |= int(z[i, w]) << (64 * w)
            kx |= int(x[i, w]) << (64 * w)
        out.append((kz, kx))
    return out


def qubit_mask(N, qubits):
    """_qubit_mask (channels.jl:14-28); raises ArgumentError for an index outside 1:N."""
    from .errors import ArgumentError
    if qubits is None:
        return (1 << N) - 1 if N > 0 else 0
    if isinstance(qubits, (int, np.integer)):
        qubits = [int(qubits)]
    m = 0
    for q in qubits:
        q = int(q)
        if not (1 <= q <= N):
            raise ArgumentError(f"qubit index {q} out of range 1:{N}")
        m |= 1 << (q - 1)
    return m
