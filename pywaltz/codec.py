"""``compress`` / ``decompress`` with the signatures and errors of the
reference's CPU bindings (python/pywaltz/codec.py:65-98 of the reference
project), computed by the GPU codec. Archives are the canonical native
archives, byte-identical to the reference CPU codec's for the same array and
bound, so files written by either side decode on the other."""

import math
import operator

import numpy as np

import waltz_b200
from waltz_b200 import WaltzError


def _geometry(shape, dtype):
    """(nx, ny, nz) of a (y,x) or (z,y,x) shape, and the checked dtype
    (python/pywaltz/codec.py:19-28)."""
    shape = tuple(operator.index(v) for v in shape)
    dtype = np.dtype(dtype)
    if dtype not in (np.dtype("float32"), np.dtype("float64")):
        raise TypeError("Waltz requires native float32 or float64")
    if len(shape) not in (2, 3) or min(shape) <= 0:
        raise ValueError("expected positive (y,x) or (z,y,x) dimensions")
    if math.prod(shape) * dtype.itemsize > 0xffffffff:
        raise ValueError("field exceeds the native Waltz archive limit")
    return (*reversed(shape), 1)[:3], dtype


def _bound(value):
    value = float(value)
    if not math.isfinite(value) or value <= 0:
        raise ValueError("abs_error must be finite and positive")
    return value


def compress(array, *, abs_error):
    """Return canonical archive bytes. The input is never modified."""
    a = np.asarray(array)
    _geometry(a.shape, a.dtype)
    bound = _bound(abs_error)
    try:
        return waltz_b200.compress(a, abs_error=bound)
    except WaltzError as exc:
        raise ValueError(str(exc)) from exc


def decompress(archive, *, shape, dtype):
    """Decode bytes using the original NumPy shape and dtype (not stored together in the archive)."""
    shape = tuple(shape)
    _, dtype = _geometry(shape, dtype)
    if len(memoryview(archive).cast("B")) < 32:
        raise ValueError("truncated Waltz header")
    try:
        return waltz_b200.decompress(bytes(archive), shape=shape, dtype=dtype)
    except WaltzError as exc:
        raise ValueError(str(exc)) from exc
