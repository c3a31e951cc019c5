"""Exception classes of the Python host API (no library load).

They mirror the reference's Julia exception classes, which the C ABI reports as
status codes (include/pauliprop.h).  Kept apart from the ctypes binding so that
the host-side strategy, Pauli-string and circuit modules import without loading
libpauliprop.so.
"""


class ArgumentError(ValueError):
    """Julia ArgumentError (bad probability, qubit index, window, strategy kind)."""


class DimensionMismatch(ValueError):
    """Julia DimensionMismatch (generators and angles of different length)."""


class PauliPropError(RuntimeError):
    """Julia ErrorException (N > 128, complex coefficient for real storage, broken invariant)."""


class DeviceError(RuntimeError):
    """CUDA runtime failure, or no CUDA device present."""
