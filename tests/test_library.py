"""The CUDA library builds, loads without a GPU, and exports every entry
point that include/*.h declares (no compute calls here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


# The HDF5 filter plugin is its own library (waltz_b200/plugins/libwaltz_h5z.so).
PLUGIN_HEADERS = {"waltz_h5z.h"}


def declared_functions(headers=None):
    names = set()
    for header in sorted((ROOT / "include").glob("*.h")):
        if (header.name in PLUGIN_HEADERS) != (headers == "plugin"):
            continue
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        for m in re.finditer(r"\b([a-z_][a-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith("waltz_") and not name.endswith("_t"):
                names.add(name)
    return names


def test_headers_declare_the_reference_entry_points():
    names = declared_functions()
    assert {"waltz_cuda_decode_chunk", "waltz_gpu_decode_batch", "waltz_b200_compress",
            "waltz_b200_decompress", "waltz_b200_extrema", "waltz_b200_compressed_capacity"} <= names


def test_library_loads_and_exports_every_declared_symbol():
    from waltz_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_plugin_exports_every_declared_symbol():
    from waltz_b200 import build
    build.build()
    lib = ctypes.CDLL(str(build.PLUGIN))
    names = declared_functions("plugin")
    assert names == {"waltz_b200_h5z_filter"}
    assert all(hasattr(lib, n) for n in names | {"H5PLget_plugin_type", "H5PLget_plugin_info"})


def test_binding_covers_every_declared_symbol():
    from waltz_b200 import _lib
    assert declared_functions() <= set(_lib.SIGNATURES)


def test_capacity_matches_reference_formula():
    from waltz_b200 import compressed_capacity
    for n, w in [(1, 4), (1000, 8), (1 << 21, 4), (1 << 23, 8), (512 ** 3, 4)]:
        pwe, qout = min(n, 1 << 22), min(n, 1 << 20)
        assert compressed_capacity(n, w) == n * w + pwe * (4 + w) + qout * 8 + (1 << 20)


def test_api_rejects_without_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import numpy as np
    import waltz_b200
    with pytest.raises(waltz_b200.WaltzError):
        waltz_b200.compress(np.zeros((4, 4, 4), np.float32), abs_error=1e-3)


def test_noalloc_encoder_host_checks_without_a_device():
    """The allocation-free WZP encoder refuses bad arguments on the host,
    before it touches a device: null pointers, an empty input, unaligned
    magnitudes and inputs beyond its static array (16384 chunks of 8192
    magnitudes). The pointers are never dereferenced on these paths."""
    from waltz_b200 import _lib
    lib = _lib.lib()
    fn = lib.waltz_b200_wzp_encode_noalloc
    base = 0x10000  # a 16-byte aligned stand-in address
    cases = [
        ((None, base, 64, base, 1 << 20), "null argument"),
        ((base, base, 0, base, 1 << 20), "must be positive"),
        ((base + 2, base, 64, base, 1 << 20), "16-byte aligned"),
        ((base, base, 16384 * 8192 + 1, base, 1 << 30), "allocation-free limit"),
    ]
    for (dm, ds, n, out, cap), message in cases:
        written = ctypes.c_size_t(7)
        rc = fn(ctypes.c_void_p(dm), ctypes.c_void_p(ds), ctypes.c_uint32(n), ctypes.c_void_p(out),
                ctypes.c_size_t(cap), ctypes.byref(written), None)
        assert rc != 0
        assert message in _lib.last_error()
        if dm is not None:
            assert written.value == 0
