"""ctypes access to the CPU checkers. TEST INFRASTRUCTURE ONLY.

Two libraries live here:

* ``liboracle.so`` -- the plain-C restatement of the reference CPU scalar
  codec (waltz_oracle.c). Built by ``make -C oracle`` (gcc is enough), on
  demand when missing.
* ``_ref/libwaltz_ref.so`` -- the reference CPU codec compiled from its own
  sources (``make -C oracle ref``); present only where the reference sources
  were available when it was built.
* ``_ref/libwaltz_refgpu.so`` -- the reference's own CUDA library compiled for
  sm_100a from its sources (``make -C oracle refgpu``): a second checker on the
  GPU (its archives must equal the product's) and the same-GPU baseline.

Only tests/, ``__graft_entry__.smoke()`` and the baseline legs of
``bench.py`` import this module, and only as the checker or the baseline.
The GPU product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libwaltz_ref.so"
REFGPU_SO = HERE / "_ref" / "libwaltz_refgpu.so"


class WoConfig(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("width", C.c_int), ("abs_error", C.c_double)]


class RefConfig(C.Structure):
    # waltz_cpu_config of the reference (cpu/include/waltz_cpu.h:13-18)
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("type", C.c_int), ("absolute_error", C.c_double), ("backend", C.c_int)]


SCALAR, AVX2 = 1, 2


def build_oracle() -> Path:
    """Compile liboracle.so if it is missing or older than its sources."""
    srcs = [HERE / "waltz_oracle.c", HERE / "waltz_oracle.h", HERE / "waltz_oracle_real.inc"]
    if not ORACLE_SO.exists() or any(s.stat().st_mtime > ORACLE_SO.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    return ORACLE_SO


@lru_cache(maxsize=1)
def oracle_lib():
    lib = C.CDLL(str(build_oracle()))
    p, sz, u32 = C.c_void_p, C.c_size_t, C.c_uint32
    sig = {
        "wo_levels": (C.c_uint, [u32]),
        "wo_zband": (C.c_uint, [u32, u32, u32, C.c_uint, C.c_int]),
        "wo_morton": (u32, [u32] * 6),
        "wo_transform": (C.c_int, [p, C.c_int, u32, u32, u32, C.c_uint, C.c_uint, C.c_int, C.c_int]),
        "wo_wzp_max_bytes": (sz, [u32]),
        "wo_wzp_encode": (C.c_longlong, [p, p, u32, p, sz, C.c_char_p, sz]),
        "wo_wzp_decode": (C.c_int, [p, sz, u32, p, p, C.c_char_p, sz]),
        "wo_quantize": (C.c_longlong, [p, C.c_int, u32, u32, u32, C.c_uint, C.c_double, p, p, p, p,
                                       C.c_char_p, sz]),
        "wo_max_compressed_bytes": (sz, [C.POINTER(WoConfig)]),
        "wo_compress": (C.c_int, [C.POINTER(WoConfig), p, p, sz, C.POINTER(sz), C.c_char_p, sz]),
        "wo_decompress": (C.c_int, [C.POINTER(WoConfig), p, sz, p, sz, C.c_char_p, sz]),
        "wo_compact_repairs": (C.c_int, [p, sz, C.c_int, p, C.c_double, p, sz, C.POINTER(sz), C.c_char_p, sz]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


def ref_available() -> bool:
    return REF_SO.exists()


@lru_cache(maxsize=1)
def ref_lib():
    if not REF_SO.exists():
        raise FileNotFoundError("reference CPU codec not built (make -C oracle ref)")
    lib = C.CDLL(str(REF_SO))
    p, sz = C.c_void_p, C.c_size_t
    cfg = C.POINTER(RefConfig)
    sig = {
        "waltz_cpu_create": (p, []), "waltz_cpu_destroy": (None, [p]),
        "waltz_cpu_last_error": (C.c_char_p, [p]),
        "waltz_cpu_max_compressed_bytes": (sz, [cfg]),
        "waltz_cpu_compress": (C.c_int, [p, cfg, p, p, sz, C.POINTER(sz)]),
        "waltz_cpu_decompress": (C.c_int, [p, cfg, p, sz, p, sz]),
        "waltz_cpu_has_avx2": (C.c_int, []),
        "ref_last_error": (C.c_char_p, []),
        "ref_transform": (C.c_int, [p, p, C.c_int] + [C.c_uint] * 5 + [C.c_int] * 3),
        "ref_transform_scratch_elements": (sz, [C.c_uint] * 3),
        "ref_wzp_max_bytes": (sz, [C.c_uint]),
        "ref_wzp_encode": (C.c_longlong, [p, p, C.c_uint, p, sz, C.c_int]),
        "ref_wzp_decode": (C.c_int, [p, sz, C.c_uint, p, p, C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


def refgpu_available() -> bool:
    return REFGPU_SO.exists()


@lru_cache(maxsize=1)
def refgpu_lib():
    """The reference CUDA library (device pointers; see ref_gpu_shim.cu)."""
    if not REFGPU_SO.exists():
        raise FileNotFoundError("reference CUDA library not built (make -C oracle refgpu)")
    lib = C.CDLL(str(REFGPU_SO))
    p, u32 = C.c_void_p, C.c_uint32
    sig = {
        "refgpu_last_error": (C.c_char_p, []),
        "refgpu_report": (None, [C.c_int]),
        "refgpu_capacity": (C.c_size_t, [C.c_uint64, C.c_int]),
        "refgpu_compress": (C.c_int, [p, C.c_int, u32, u32, u32, C.c_double, p, C.POINTER(C.c_size_t), p]),
        "refgpu_decompress": (C.c_int, [p, C.c_int, u32, u32, u32, p, p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


def refgpu_compress(d_in: int, width: int, shape, abs_error: float, d_out: int, stream: int) -> int:
    """Archive bytes the reference CUDA library writes at d_out (device
    pointers, (z, y, x) shape)."""
    nz, ny, nx = shape
    w = C.c_size_t()
    lib = refgpu_lib()
    if lib.refgpu_compress(C.c_void_p(d_in), width, nx, ny, nz, abs_error, C.c_void_p(d_out), C.byref(w),
                           C.c_void_p(stream)):
        raise RuntimeError(lib.refgpu_last_error().decode())
    return w.value


def refgpu_decompress(d_archive: int, width: int, shape, d_out: int, stream: int) -> None:
    nz, ny, nx = shape
    lib = refgpu_lib()
    if lib.refgpu_decompress(C.c_void_p(d_archive), width, nx, ny, nz, C.c_void_p(d_out), C.c_void_p(stream)):
        raise RuntimeError(lib.refgpu_last_error().decode())


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _dims(shape):
    """numpy (z,y,x) shape -> (nx, ny, nz)."""
    nz, ny, nx = shape
    return nx, ny, nz


class CodecError(ValueError):
    pass


# ------------------------------------------------------------------ oracle

def levels(n: int) -> int:
    return int(oracle_lib().wo_levels(n))


def zband(nx, ny, nz, lz, dyadic) -> int:
    return int(oracle_lib().wo_zband(nx, ny, nz, lz, int(dyadic)))


def transform(field: np.ndarray, *, inverse: bool, lxy=None, lz=None, dyadic=None) -> np.ndarray:
    """All-level transform of a (z,y,x) array (a copy is returned)."""
    out = np.ascontiguousarray(field).copy()
    nx, ny, nz = _dims(out.shape)
    if lxy is None:
        lxy, lz = levels(min(nx, ny)), levels(nz)
        dyadic = lxy == lz
    if oracle_lib().wo_transform(_ptr(out), out.itemsize, nx, ny, nz, lxy, lz, int(dyadic), int(inverse)):
        raise CodecError("invalid transform arguments")
    return out


def wzp_encode(mag: np.ndarray, sign: np.ndarray) -> bytes:
    n = mag.size
    lib = oracle_lib()
    out = np.zeros(max(lib.wo_wzp_max_bytes(n), 1), np.uint8)
    err = C.create_string_buffer(256)
    r = lib.wo_wzp_encode(_ptr(mag), _ptr(sign), n, _ptr(out), out.size, err, 256)
    if r < 0:
        raise CodecError(err.value.decode())
    return out[:r].tobytes()


def wzp_decode(stream: bytes, n: int):
    src = np.frombuffer(stream, np.uint8).copy() if stream else np.zeros(1, np.uint8)
    mag = np.zeros(max(n, 1), np.uint16)
    sign = np.zeros(max((n + 31) // 32, 1), np.uint32)
    err = C.create_string_buffer(256)
    if oracle_lib().wo_wzp_decode(_ptr(src), len(stream), n, _ptr(mag), _ptr(sign), err, 256):
        raise CodecError(err.value.decode())
    return mag[:n], sign[:(n + 31) // 32]


def quantize(coeff: np.ndarray, bz: int, quantum: float):
    """Quantise a transformed (z,y,x) array; returns (dequantised, mag, sign, qidx, qval)."""
    data = np.ascontiguousarray(coeff).copy()
    n = data.size
    nx, ny, nz = _dims(data.shape)
    mag = np.zeros(n, np.uint16)
    sign = np.zeros((n + 31) // 32, np.uint32)
    qidx = np.zeros(n, np.uint32)
    qval = np.zeros(n, np.uint32)
    err = C.create_string_buffer(256)
    r = oracle_lib().wo_quantize(_ptr(data), data.itemsize, nx, ny, nz, bz, quantum,
                                 _ptr(mag), _ptr(sign), _ptr(qidx), _ptr(qval), err, 256)
    if r < 0:
        raise CodecError(err.value.decode())
    return data, mag, sign, qidx[:r].copy(), qval[:r].copy()


def max_compressed_bytes(shape, dtype, abs_error=1.0) -> int:
    nx, ny, nz = _dims(shape)
    cfg = WoConfig(nx, ny, nz, np.dtype(dtype).itemsize, abs_error)
    return int(oracle_lib().wo_max_compressed_bytes(C.byref(cfg)))


def compress(field: np.ndarray, abs_error: float) -> bytes:
    a = np.ascontiguousarray(field)
    nx, ny, nz = _dims(a.shape)
    cfg = WoConfig(nx, ny, nz, a.itemsize, abs_error)
    lib = oracle_lib()
    cap = lib.wo_max_compressed_bytes(C.byref(cfg))
    if not cap:
        raise CodecError("unsupported configuration")
    out = np.zeros(cap, np.uint8)
    written = C.c_size_t()
    err = C.create_string_buffer(256)
    if lib.wo_compress(C.byref(cfg), _ptr(a), _ptr(out), cap, C.byref(written), err, 256):
        raise CodecError(err.value.decode())
    return out[:written.value].tobytes()


def decompress(archive: bytes, shape, dtype) -> np.ndarray:
    out = np.zeros(shape, dtype)
    nx, ny, nz = _dims(shape)
    cfg = WoConfig(nx, ny, nz, out.itemsize, 0.0)
    src = np.frombuffer(archive, np.uint8).copy() if archive else np.zeros(1, np.uint8)
    err = C.create_string_buffer(256)
    if oracle_lib().wo_decompress(C.byref(cfg), _ptr(src), len(archive), _ptr(out), out.nbytes, err, 256):
        raise CodecError(err.value.decode())
    return out


def compact_repairs(archive: bytes, field: np.ndarray, step: float) -> bytes:
    """The archive with its repair section in the compact WPW1 form (groups in
    order, as the GPU encoder writes it) where that is smaller, else itself."""
    a = np.ascontiguousarray(field)
    src = np.frombuffer(archive, np.uint8).copy()
    out = np.zeros(len(archive), np.uint8)
    written = C.c_size_t()
    err = C.create_string_buffer(256)
    if oracle_lib().wo_compact_repairs(_ptr(src), len(archive), a.itemsize, _ptr(a), step, _ptr(out), out.size,
                                       C.byref(written), err, 256):
        raise CodecError(err.value.decode())
    return out[:written.value].tobytes()


# --------------------------------------------------------------- reference

class RefCodec:
    """The reference CPU codec (scalar or AVX2 backend) through its C API."""

    def __init__(self, backend: int = SCALAR):
        self.lib = ref_lib()
        self.backend = backend
        self.ws = self.lib.waltz_cpu_create()

    def __del__(self):
        try:
            self.lib.waltz_cpu_destroy(self.ws)
        except Exception:
            pass

    def _cfg(self, shape, dtype, abs_error):
        nx, ny, nz = _dims(shape)
        return RefConfig(nx, ny, nz, np.dtype(dtype).itemsize, abs_error, self.backend)

    def compress(self, field: np.ndarray, abs_error: float) -> bytes:
        a = np.ascontiguousarray(field)
        cfg = self._cfg(a.shape, a.dtype, abs_error)
        cap = self.lib.waltz_cpu_max_compressed_bytes(C.byref(cfg))
        out = np.zeros(max(cap, 1), np.uint8)
        written = C.c_size_t()
        if self.lib.waltz_cpu_compress(self.ws, C.byref(cfg), _ptr(a), _ptr(out), cap, C.byref(written)):
            raise CodecError(self.lib.waltz_cpu_last_error(self.ws).decode())
        return out[:written.value].tobytes()

    def decompress(self, archive: bytes, shape, dtype) -> np.ndarray:
        out = np.zeros(shape, dtype)
        cfg = self._cfg(shape, dtype, 0.0)
        src = np.frombuffer(archive, np.uint8).copy() if archive else np.zeros(1, np.uint8)
        if self.lib.waltz_cpu_decompress(self.ws, C.byref(cfg), _ptr(src), len(archive), _ptr(out), out.nbytes):
            raise CodecError(self.lib.waltz_cpu_last_error(self.ws).decode())
        return out


def ref_transform(field: np.ndarray, *, inverse: bool, avx2: bool = False) -> np.ndarray:
    lib = ref_lib()
    out = np.ascontiguousarray(field).copy()
    nx, ny, nz = _dims(out.shape)
    lxy, lz = levels(min(nx, ny)), levels(nz)
    scratch = np.zeros(lib.ref_transform_scratch_elements(nx, ny, nz), out.dtype)
    if lib.ref_transform(_ptr(out), _ptr(scratch), out.itemsize, nx, ny, nz, lxy, lz,
                         int(lxy == lz), int(inverse), int(avx2)):
        raise CodecError(lib.ref_last_error().decode())
    return out


def ref_wzp_encode(mag: np.ndarray, sign: np.ndarray, avx2: bool = False) -> bytes:
    lib = ref_lib()
    n = mag.size
    out = np.zeros(max(lib.ref_wzp_max_bytes(n), 1), np.uint8)
    r = lib.ref_wzp_encode(_ptr(mag), _ptr(sign), n, _ptr(out), out.size, int(avx2))
    if r < 0:
        raise CodecError(lib.ref_last_error().decode())
    return out[:r].tobytes()


def ref_wzp_decode(stream: bytes, n: int):
    lib = ref_lib()
    src = np.frombuffer(stream, np.uint8).copy() if stream else np.zeros(1, np.uint8)
    mag = np.zeros(max(n, 1), np.uint16)
    sign = np.zeros(max((n + 31) // 32, 1), np.uint32)
    if lib.ref_wzp_decode(_ptr(src), len(stream), n, _ptr(mag), _ptr(sign), 0):
        raise CodecError(lib.ref_last_error().decode())
    return mag[:n], sign[:(n + 31) // 32]
