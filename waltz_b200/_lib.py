"""ctypes binding of the in-tree CUDA library ``libwaltz_b200.so``.

The library is the only compute path: if it is missing or cannot load, every
call raises. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from functools import lru_cache
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libwaltz_b200.so"


class BatchShape(C.Structure):
    """waltz_batch_shape (include/waltz_gpu_batch.h)."""
    _fields_ = [(name, C.c_uint32) for name in ("x", "y", "z", "fx", "fy", "fz", "samples", "sides", "width")]


# exported name -> (restype, argtypes); mirrors include/*.h
SIGNATURES = {
    "waltz_b200_compressed_capacity": (C.c_size_t, [C.c_uint64, C.c_int]),
    "waltz_b200_compress": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                      C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_void_p]),
    "waltz_b200_compress_form": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                           C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_void_p]),
    "waltz_b200_compress_batch": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_uint64), C.c_void_p]),
    "waltz_b200_batch_config": (C.c_int, [C.c_int, C.c_int]),
    "waltz_b200_set_option": (C.c_int, [C.c_int, C.c_int]),
    "waltz_b200_decompress_batch": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]),
    "waltz_b200_decompress": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.c_void_p, C.c_size_t, C.c_void_p]),
    "waltz_b200_extrema": (C.c_int, [C.c_void_p, C.c_int, C.c_uint64, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.c_void_p]),
    "waltz_b200_last_error": (C.c_char_p, []),
    "waltz_b200_transform": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                                       C.c_void_p]),
    "waltz_b200_wzp_encode": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t,
                                        C.POINTER(C.c_size_t), C.c_void_p]),
    "waltz_b200_zmatrix": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]),
    "waltz_b200_zmatrix_f64": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]),
    "waltz_b200_zmatrix_split": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int,
                                           C.c_void_p]),
    "waltz_b200_wzp_encode_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t,
                                                C.POINTER(C.c_size_t), C.c_void_p]),
    "waltz_b200_test_lookback_timeout": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32,
                                                   C.c_double, C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint32,
                                                   C.c_void_p]),
    "waltz_b200_launch_count": (C.c_ulonglong, []),
    "waltz_b200_graph_count": (C.c_ulonglong, []),
    "waltz_b200_profile": (None, [C.c_int]),
    "waltz_b200_stage_times": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_char_p), C.c_int]),
    "waltz_cuda_decode_chunk": (C.c_char_p, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p,
                                             C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p]),
    "waltz_gpu_decode_batch": (C.c_char_p, [C.POINTER(BatchShape), C.c_void_p, C.c_void_p, C.c_size_t,
                                            C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_double,
                                            C.c_void_p]),
}


class Chunk(C.Structure):
    """waltz_b200_chunk (include/waltz_b200.h)."""
    _fields_ = [("input", C.c_void_p), ("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("abs_error", C.c_double), ("archive", C.c_void_p), ("capacity", C.c_uint64)]


class Archive(C.Structure):
    """waltz_b200_archive (include/waltz_b200.h)."""
    _fields_ = [("archive", C.c_void_p), ("bytes", C.c_uint64), ("header", C.c_void_p), ("nx", C.c_uint32),
                ("ny", C.c_uint32), ("nz", C.c_uint32), ("output", C.c_void_p), ("output_bytes", C.c_uint64),
                ("stride_y", C.c_uint64), ("stride_z", C.c_uint64)]


class WaltzError(RuntimeError):
    pass


@lru_cache(maxsize=1)
def lib():
    path = Path(os.environ.get("WALTZ_B200_LIBRARY", LIB_PATH))
    if not path.exists():
        raise WaltzError(f"CUDA library {path} is missing: run `python -m waltz_b200.build` "
                         "(there is no CPU fallback)")
    handle = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype, fn.argtypes = res, args
    return handle


def last_error() -> str:
    msg = lib().waltz_b200_last_error()
    return msg.decode(errors="replace") if msg else "unknown error"


def checked(rc: int) -> None:
    if rc != 0:
        raise WaltzError(last_error())
