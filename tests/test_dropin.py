"""The drop-in surfaces without a GPU: the C++ device API's exported names
and Config layout against the reference's, the HDF5 filter plugin's entry
points and argument checks, and the pywaltz shim's argument errors. No
compute call runs here."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CALLERS = {"ours": ROOT / "tests" / "cxx" / "libcaller.so",
           "reference header": ROOT / "tests" / "cxx" / "libcaller_refhdr.so"}
REFGPU = ROOT / "oracle" / "_ref" / "libwaltz_refgpu.so"

CXX_ENTRY_POINTS = [
    "_ZN5WALTZ16d_WALTZ_compressIfLi3EEEmPT_PcRKNS_6ConfigEPKcPv",
    "_ZN5WALTZ16d_WALTZ_compressIdLi3EEEmPT_PcRKNS_6ConfigEPKcPv",
    "_ZN5WALTZ18d_WALTZ_decompressIfLi3EEEmPcPT_RKNS_6ConfigEPKcPv",
    "_ZN5WALTZ18d_WALTZ_decompressIdLi3EEEmPcPT_RKNS_6ConfigEPKcPv",
    "_ZN5WALTZ9d_extremaIfEEvPT_mRdS3_Pv",
    "_ZN5WALTZ9d_extremaIdEEvPT_mRdS3_Pv",
    "_ZN5WALTZ20calculate_dwt_levelsE4dim3RhS1_",
]


def _exports(path: Path) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], check=True, capture_output=True, text=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}


def _build():
    from waltz_b200 import build
    build.build()
    subprocess.run(["make", "-s", "-C", str(ROOT / "tests" / "cxx"), "all"], check=True)


def test_library_exports_the_reference_cxx_entry_points():
    _build()
    from waltz_b200 import build
    exported = _exports(build.LIB)
    assert set(CXX_ENTRY_POINTS) <= exported
    if REFGPU.exists():
        # every C++ API entry point the reference's own library exports is here too
        ref = {s for s in _exports(REFGPU)
               if s.startswith(("_ZN5WALTZ16d_WALTZ_", "_ZN5WALTZ18d_WALTZ_", "_ZN5WALTZ9d_extrema",
                                "_ZN5WALTZ20calculate_dwt"))}
        assert ref and ref <= exported, sorted(ref - exported)


def _caller(name):
    path = CALLERS[name]
    if not path.exists():
        pytest.skip(f"{path.name} is built only where the reference tree is present")
    return C.CDLL(str(path))


@pytest.mark.parametrize("name", list(CALLERS))
def test_config_layout_and_helpers(name):
    _build()
    lib = _caller(name)
    layout = (C.c_ulonglong * 8)()
    assert lib.caller_config_layout(layout, 8) == 8
    # ndims, dimx, dimy, dimz, num, errorBoundMode, absErrorBound, sizeof
    assert list(layout) == [0, 8, 16, 24, 72, 88, 96, 128]
    dims = (C.c_ulonglong * 5)()
    lib.caller_config_dims(C.c_ulonglong(64), C.c_ulonglong(1), C.c_ulonglong(32), dims)
    assert list(dims) == [2, 64, 32, 1, 64 * 32]  # extents of 1 are dropped
    lib.caller_config_dims(C.c_ulonglong(96), C.c_ulonglong(40), C.c_ulonglong(24), dims)
    assert list(dims) == [3, 96, 40, 24, 96 * 40 * 24]
    lib.caller_capacity_f32.restype = lib.caller_capacity_f64.restype = C.c_ulonglong
    from waltz_b200 import compressed_capacity
    for n in (1, 1000, 1 << 21, 512 ** 3):
        assert lib.caller_capacity_f32(C.c_ulonglong(n)) == compressed_capacity(n, 4)
        assert lib.caller_capacity_f64(C.c_ulonglong(n)) == compressed_capacity(n, 8)
    from oracle import oracle as O
    lxy, lz = C.c_ubyte(), C.c_ubyte()
    for x, y, z in [(64, 64, 64), (1024, 1024, 64), (384, 256, 96), (9, 300, 5), (1, 1, 1)]:
        lib.caller_levels(x, y, z, C.byref(lxy), C.byref(lz))
        assert (lxy.value, lz.value) == (O.levels(min(x, y)), O.levels(z))


# ------------------------------------------------------------------ HDF5 plugin

class FilterClass(C.Structure):
    """H5Z_class2_t."""
    _fields_ = [("version", C.c_int), ("id", C.c_int), ("encoder_present", C.c_uint),
                ("decoder_present", C.c_uint), ("name", C.c_char_p), ("can_apply", C.c_void_p),
                ("set_local", C.c_void_p), ("filter", C.c_void_p)]


FILTER_FN = C.CFUNCTYPE(C.c_size_t, C.c_uint, C.c_size_t, C.POINTER(C.c_uint), C.c_size_t,
                        C.POINTER(C.c_size_t), C.POINTER(C.c_void_p))


def plugin():
    from waltz_b200 import build
    build.build()
    lib = C.CDLL(str(build.PLUGIN))
    lib.H5PLget_plugin_type.restype = C.c_int
    lib.H5PLget_plugin_info.restype = C.POINTER(FilterClass)
    return lib


def test_h5z_plugin_entry_points():
    lib = plugin()
    assert lib.H5PLget_plugin_type() == 0  # H5PL_TYPE_FILTER
    info = lib.H5PLget_plugin_info().contents
    assert (info.version, info.id, info.encoder_present, info.decoder_present) == (1, 61197, 1, 1)
    assert info.name.startswith(b"Waltz canonical")
    assert info.can_apply is None and info.set_local is None and info.filter
    assert C.cast(lib.waltz_b200_h5z_filter, C.c_void_p).value == info.filter


def test_h5z_filter_rejects_bad_arguments_untouched():
    """Argument checks run before any device work and leave the buffer as it
    was (python/hdf5/filter.cpp:19-36 of the reference)."""
    from pywaltz.hdf5 import filter_values
    lib = plugin()
    fn = FILTER_FN(C.cast(lib.H5PLget_plugin_info().contents.filter, C.c_void_p).value)
    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    libc.free.argtypes = [C.c_void_p]
    good = filter_values((8, 16, 16), np.float32, 1e-3)
    raw = 8 * 16 * 16 * 4
    cases = [
        (0, 5, good, raw, raw),                               # wrong client-data count
        (0, 6, (16, 16, 8, 3, *good[4:]), raw, raw),          # width neither 4 nor 8
        (0, 6, good, raw - 4, raw),                           # forward size is not the chunk
        (0, 6, good, raw, raw - 8),                           # bytes beyond the buffer
        (0, 6, (0, 16, 8, 4, *good[4:]), raw, raw),           # empty extent
        (0, 6, (*good[:4], 0, 0), raw, raw),                  # bound 0
        (0x0100, 6, good, 16, raw),                           # archive shorter than its header
        (0x0100, 6, good, 1 << 40, 1 << 41),                  # archive beyond the capacity
    ]
    for flags, count, cd, nbytes, size in cases:
        ptr = libc.malloc(64)
        buf = C.c_void_p(ptr)
        bsize = C.c_size_t(size)
        words = (C.c_uint * 6)(*cd)
        assert fn(flags, count, words, nbytes, C.byref(bsize), C.byref(buf)) == 0
        assert buf.value == ptr and bsize.value == size
        libc.free(ptr)


def test_h5z_filter_values_match_the_reference_layout():
    import struct
    from pywaltz.hdf5 import FILTER_ID, filter_values
    assert FILTER_ID == 61197
    lo, hi = struct.unpack("<II", struct.pack("<d", 2.5e-4))
    assert filter_values((12, 34, 56), np.float64, 2.5e-4) == (56, 34, 12, 8, lo, hi)
    assert filter_values((34, 56), np.float32, 2.5e-4) == (56, 34, 1, 4, lo, hi)


# ------------------------------------------------------------------ pywaltz shim

def test_pywaltz_argument_errors_match_the_reference():
    import pywaltz
    with pytest.raises(TypeError):
        pywaltz.compress(np.zeros((4, 4, 4), np.int32), abs_error=1e-3)
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(ValueError):
            pywaltz.compress(np.zeros((4, 4, 4), np.float32), abs_error=bad)
    with pytest.raises(ValueError):
        pywaltz.compress(np.zeros((4,), np.float32), abs_error=1e-3)
    with pytest.raises(ValueError):
        pywaltz.decompress(b"\0" * 16, shape=(4, 4, 4), dtype=np.float32)
    with pytest.raises(TypeError):
        pywaltz.decompress(b"\0" * 64, shape=(4, 4, 4), dtype=np.int16)
