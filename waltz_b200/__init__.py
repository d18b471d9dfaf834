"""Waltz error-bounded 3-D compressor, B200-native.

Host-side mirror of the reference's Python surface (python/pywaltz/codec.py:
``compress(array, *, abs_error)`` / ``decompress(archive, *, shape, dtype)``),
running on the GPU through the in-tree CUDA library, plus device-tensor
entry points for callers whose data already lives in HBM. Archives are the
reference's native 32-byte-header archives, byte-identical to the reference
CPU scalar codec in the default profile.
"""
from __future__ import annotations

import ctypes as C
import math
import operator

import numpy as np

from . import autotune
from ._lib import Archive, BatchShape, Chunk, WaltzError, checked, lib

__all__ = ["compress", "decompress", "compress_tensor", "decompress_tensor", "compress_batch", "decompress_batch", "extrema",
           "compressed_capacity", "rel_to_abs_bound", "WaltzError"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise WaltzError("a CUDA device is required (there is no CPU fallback)")
    return torch


def _geometry(shape, itemsize):
    """(z,y,x) or (y,x) shape -> (nx, ny, nz), as python/pywaltz/codec.py:24-33."""
    shape = tuple(operator.index(v) for v in shape)
    if itemsize not in (4, 8):
        raise TypeError("Waltz requires native float32 or float64")
    if len(shape) not in (2, 3) or min(shape) <= 0:
        raise ValueError("expected positive (y,x) or (z,y,x) dimensions")
    if math.prod(shape) * itemsize > 0xffffffff:
        raise ValueError("field exceeds the native Waltz archive limit")
    return (*reversed(shape), 1)[:3]


def _bound(value):
    value = float(value)
    if not math.isfinite(value) or value <= 0:
        raise ValueError("abs_error must be finite and positive")
    return value


def compressed_capacity(n: int, itemsize: int) -> int:
    return int(lib().waltz_b200_compressed_capacity(n, itemsize))


def _stream(torch, stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


# Transform forms: the default lifting profile, and the precision form's
# tensor-core splits (include/waltz_b200.h, WALTZ_B200_FORM_*).
FORMS = {"plain": 0, "matrix": 1, "matrix-tf32": 1, "matrix-bf16": 2, "matrix-exact": 3}


def _matrix_ok(shape, itemsize, form="matrix"):
    nx, ny, nz = _geometry(shape, itemsize)
    lxy, lz = (autotune._levels(min(nx, ny)), autotune._levels(nz))
    kmax = 96 if form == "matrix-exact" else 128
    return itemsize in (4, 8) and lxy != lz and lz >= 1 and nz <= kmax and (nx * ny) % 4 == 0


def auto_form(shape, itemsize):
    """The form form="auto" takes: the precision-form split the tuning table
    chose for the field's class (the fastest split that beat the plain form
    by 3 % with an archive within 2 % of the plain one's size), where the
    matrix form applies to this field; the plain form elsewhere."""
    if not _matrix_ok(shape, itemsize):
        return "plain"
    form = autotune.matrix_choice(tuple(shape), itemsize)
    return form if form and _matrix_ok(shape, itemsize, form) else "plain"


def compress_tensor(field, abs_error: float, *, form: str = "plain", stream=None, tuned=True):
    """Compress a contiguous float32/float64 CUDA tensor of shape (z,y,x) or
    (y,x). Returns a uint8 CUDA tensor holding the archive.

    form="plain" is the default profile (byte-identical to the reference CPU
    codec); form="matrix" (TF32x3), "matrix-bf16" (BF16x3) and
    "matrix-exact" (exact bf16 slices, nz <= 96) are the precision form,
    whose Z stage runs as one matrix on the tensor cores (plane schedule,
    nz <= 128); form="auto" takes auto_form(). With `tuned`, the tuning
    table's knobs for the field's class are applied first (they never change
    the output)."""
    torch = _torch()
    if not field.is_cuda or not field.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    if form not in FORMS and form != "auto":
        raise ValueError(f"form must be one of {sorted(FORMS) + ['auto']}")
    itemsize = field.element_size()
    if form == "auto":
        form = auto_form(tuple(field.shape), itemsize)
    if tuned:
        autotune.apply_single(lib(), tuple(_geometry(field.shape, itemsize))[::-1], itemsize)
    nx, ny, nz = _geometry(field.shape, field.element_size())
    cap = compressed_capacity(field.numel(), field.element_size())
    out = torch.empty(cap, dtype=torch.uint8, device=field.device)
    written = C.c_size_t()
    checked(lib().waltz_b200_compress_form(C.c_void_p(field.data_ptr()), field.element_size(), nx, ny, nz,
                                           _bound(abs_error), FORMS[form], C.c_void_p(out.data_ptr()), cap,
                                           C.byref(written), _stream(torch, stream)))
    return out[:written.value]


def decompress_tensor(archive, shape, dtype, *, out=None, stream=None, tuned=True):
    """Decode a uint8 CUDA tensor archive into a (z,y,x) CUDA tensor."""
    torch = _torch()
    dtype = {np.float32: torch.float32, np.float64: torch.float64}.get(dtype, dtype)
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("Waltz requires float32 or float64")
    itemsize = 4 if dtype == torch.float32 else 8
    nx, ny, nz = _geometry(shape, itemsize)
    if tuned:
        autotune.apply_single(lib(), (nz, ny, nx), itemsize)
    if out is None:
        out = torch.empty(tuple(shape), dtype=dtype, device=archive.device)
    if not archive.is_cuda or not archive.is_contiguous():
        raise ValueError("expected a contiguous CUDA archive tensor")
    checked(lib().waltz_b200_decompress(C.c_void_p(archive.data_ptr()), archive.numel(), itemsize, nx, ny, nz,
                                        C.c_void_p(out.data_ptr()), out.numel() * itemsize,
                                        _stream(torch, stream)))
    return out


def compress_batch(fields, abs_errors, *, out=None, stream=None, tuned=True):
    """Compress many contiguous CUDA tensors (one dtype, any shapes) in one
    call: one CUDA graph, kept and replayed while the fields, bounds and
    output buffer stay the same. Returns one uint8 archive tensor per field,
    views into `out` (a uint8 CUDA tensor; allocated when not given — pass the
    same one again to replay the graph). Every archive equals compress_tensor
    of its field."""
    torch = _torch()
    fields = list(fields)
    if not fields:
        return []
    itemsize = fields[0].element_size()
    if any(f.element_size() != itemsize or not f.is_cuda or not f.is_contiguous() for f in fields):
        raise ValueError("expected contiguous CUDA tensors of one dtype")
    bounds = [abs_errors] * len(fields) if not hasattr(abs_errors, "__len__") else list(abs_errors)
    if len(bounds) != len(fields):
        raise ValueError("one bound per field")
    offsets, total = [], 0
    for f in fields:
        total = (total + 15) // 16 * 16
        offsets.append(total)
        total += compressed_capacity(f.numel(), itemsize)
    if out is None:
        out = torch.empty(total, dtype=torch.uint8, device=fields[0].device)
    if out.numel() < total or out.dtype != torch.uint8:
        raise ValueError(f"out must be a uint8 CUDA tensor of at least {total} bytes")
    items = (Chunk * len(fields))()
    for k, (f, eb, off) in enumerate(zip(fields, bounds, offsets)):
        nx, ny, nz = _geometry(f.shape, itemsize)
        items[k] = Chunk(f.data_ptr(), nx, ny, nz, _bound(eb), out.data_ptr() + off,
                         compressed_capacity(f.numel(), itemsize))
    written = (C.c_uint64 * len(fields))()
    if tuned:
        autotune.apply_batch(lib(), [tuple(f.shape) for f in fields], itemsize)
    checked(lib().waltz_b200_compress_batch(items, len(fields), itemsize, written, _stream(torch, stream)))
    return [out[off:off + written[k]] for k, off in enumerate(offsets)]


def decompress_batch(archives, shapes, dtype, *, out=None, headers=None, stream=None, tuned=True):
    """Decode many archives (uint8 CUDA tensors, e.g. views of one staging
    buffer) of any shapes in one call, through one CUDA graph that is replayed
    while the shapes, forms and outputs stay the same. `out` is either one
    preallocated CUDA tensor of `dtype` holding at least the total sample count
    (each result is a (z,y,x) view of it, packed back to back) or a list of
    contiguous CUDA tensors, one per archive. `headers` optionally gives host
    copies (bytes-like, >= 32 bytes each) of the archives' headers. Returns the
    list of decoded (z,y,x) tensors."""
    torch = _torch()
    dtype = {np.float32: torch.float32, np.float64: torch.float64}.get(dtype, dtype)
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("Waltz requires float32 or float64")
    itemsize = 4 if dtype == torch.float32 else 8
    archives, shapes = list(archives), [tuple(s) for s in shapes]
    if len(archives) != len(shapes):
        raise ValueError("one shape per archive")
    if not archives:
        return []
    if any(not a.is_cuda or not a.is_contiguous() or a.dtype != torch.uint8 for a in archives):
        raise ValueError("expected contiguous uint8 CUDA archive tensors")
    sizes = [math.prod(s) for s in shapes]
    if out is None:
        out = torch.empty(sum(sizes), dtype=dtype, device=archives[0].device)
    if isinstance(out, (list, tuple)):
        views = list(out)
        if len(views) != len(archives) or any(v.dtype != dtype or not v.is_contiguous() or v.numel() < k
                                              for v, k in zip(views, sizes)):
            raise ValueError("one contiguous output tensor of the batch dtype per archive")
        views = [v.view(-1)[:k].view(s) for v, k, s in zip(views, sizes, shapes)]
    else:
        if out.dtype != dtype or not out.is_contiguous() or out.numel() < sum(sizes):
            raise ValueError(f"out must be a contiguous {dtype} tensor of at least {sum(sizes)} samples")
        flat, views, at = out.view(-1), [], 0
        for k, s in zip(sizes, shapes):
            views.append(flat[at:at + k].view(s))
            at += k
    keep = []
    items = (Archive * len(archives))()
    for k, (a, s, v) in enumerate(zip(archives, shapes, views)):
        nx, ny, nz = _geometry(s, itemsize)
        hdr = None
        if headers is not None:
            buf = C.create_string_buffer(bytes(headers[k][:32]), 32)
            keep.append(buf)
            hdr = C.cast(buf, C.c_void_p)
        items[k] = Archive(a.data_ptr(), a.numel(), hdr, nx, ny, nz, v.data_ptr(), v.numel() * itemsize)
    if tuned:
        autotune.apply_batch(lib(), shapes, itemsize)
    checked(lib().waltz_b200_decompress_batch(items, len(archives), itemsize, _stream(torch, stream)))
    return views


def extrema(field, *, stream=None):
    """(min, max) of a CUDA tensor, as doubles."""
    torch = _torch()
    lo, hi = C.c_double(), C.c_double()
    checked(lib().waltz_b200_extrema(C.c_void_p(field.data_ptr()), field.element_size(), field.numel(),
                                     C.byref(lo), C.byref(hi), _stream(torch, stream)))
    return lo.value, hi.value


def rel_to_abs_bound(field, rel: float, *, stream=None) -> float:
    """REL bound -> absolute bound: rel * (max - min) in double."""
    lo, hi = extrema(field, stream=stream)
    return float(rel) * (hi - lo)


def compress(array, *, abs_error, form="plain"):
    """Return archive bytes of a float32/float64 (z,y,x) or (y,x) numpy array,
    computed on the current CUDA device: canonical (reference-identical) in
    the default plain form, tensor-core Z stage with the matrix forms."""
    torch = _torch()
    a = np.ascontiguousarray(np.asarray(array))
    if a.dtype not in (np.float32, np.float64):
        raise TypeError("Waltz requires native float32 or float64")
    dev = torch.from_numpy(a).cuda()
    return bytes(compress_tensor(dev, abs_error, form=form).cpu().numpy().tobytes())


def decompress(archive, *, shape, dtype):
    """Decode archive bytes using the original numpy shape and dtype."""
    torch = _torch()
    src = np.frombuffer(archive, dtype=np.uint8)
    if src.size < 32:
        raise ValueError("truncated Waltz header")
    dev = torch.from_numpy(src.copy()).cuda()
    out = decompress_tensor(dev, tuple(shape), np.dtype(dtype).type)
    return out.cpu().numpy()
