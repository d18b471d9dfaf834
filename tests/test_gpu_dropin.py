"""GPU: the drop-in surfaces give the oracle's archives and decodes.

* the reference's C++ device API (WALTZ::d_compress / d_decompress /
  d_extrema) through a caller compiled against this repository's header and,
  where built, the same caller compiled against the reference's own header;
  the decoder takes no archive length;
* waltz_b200_decompress with length 0 (taken from the header);
* the HDF5 filter 61197 callback on malloc'd host buffers, against the oracle
  and against archives of the reference CPU codec;
* the pywaltz shim.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests import patterns as P

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CALLERS = {"ours": ROOT / "tests" / "cxx" / "libcaller.so",
           "reference header": ROOT / "tests" / "cxx" / "libcaller_refhdr.so"}

CASES = [((64, 64, 64), np.float32, "sin", 1e-3, 0.0),
         ((40, 44, 52), np.float64, "grf", 0.0, 1e-4),
         ((33, 200, 72), np.float32, "grf", 1e-5, 0.0),
         ((96, 256, 384), np.float64, "grf", 1e-3, 0.0)]


def _field(nxyz, dtype, kind, seed=11):
    from waltz_b200 import synthetic as S
    zyx = P.zyx(nxyz)
    if kind == "sin":
        return S.sinusoids(zyx, seed=seed, dtype=dtype)
    return S.power_law_field(zyx, seed, dtype=dtype)


def _caller(name):
    path = CALLERS[name]
    if not path.exists():
        pytest.skip(f"{path.name} is built only where the reference tree is present")
    lib = C.CDLL(str(path))
    for f in ("caller_round_trip_f32", "caller_round_trip_f64"):
        getattr(lib, f).argtypes = [C.c_void_p, C.c_ulonglong, C.c_ulonglong, C.c_ulonglong, C.c_double,
                                    C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_ulonglong),
                                    C.POINTER(C.c_double), C.c_char_p, C.c_ulonglong]
    lib.caller_decode_f32.argtypes = [C.c_void_p, C.c_ulonglong, C.c_ulonglong, C.c_ulonglong, C.c_void_p,
                                      C.c_void_p, C.c_char_p, C.c_ulonglong]
    return lib


@pytest.mark.parametrize("name", list(CALLERS))
@pytest.mark.parametrize("nxyz,dtype,kind,rel,abs_bound", CASES)
def test_cxx_api_round_trip_matches_oracle(name, nxyz, dtype, kind, rel, abs_bound):
    import torch
    from waltz_b200 import compressed_capacity
    lib = _caller(name)
    a = _field(nxyz, dtype, kind)
    d_in = torch.from_numpy(a).cuda()
    cap = compressed_capacity(a.size, a.itemsize)
    d_cmp = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    d_out = torch.empty_like(d_in)
    nbytes, bound = C.c_ulonglong(), C.c_double()
    err = C.create_string_buffer(512)
    fn = lib.caller_round_trip_f32 if dtype == np.float32 else lib.caller_round_trip_f64
    nx, ny, nz = nxyz
    rc = fn(d_in.data_ptr(), nx, ny, nz, rel, abs_bound, d_cmp.data_ptr(), d_out.data_ptr(),
            torch.cuda.current_stream().cuda_stream, C.byref(nbytes), C.byref(bound), err, 512)
    assert rc == 0, err.value.decode()
    eb = bound.value
    if rel:
        assert eb == rel * (float(a.max()) - float(a.min()))
    archive = d_cmp[:nbytes.value].cpu().numpy().tobytes()
    assert archive == O.compress(a, eb)
    assert d_out.cpu().numpy().tobytes() == O.decompress(archive, a.shape, dtype).tobytes()


@pytest.mark.parametrize("name", list(CALLERS))
def test_cxx_api_errors_are_exceptions(name):
    import torch
    from waltz_b200 import compressed_capacity
    lib = _caller(name)
    a = _field((32, 32, 32), np.float32, "grf")
    d_in = torch.from_numpy(a).cuda()
    d_cmp = torch.zeros(compressed_capacity(a.size, 4), dtype=torch.uint8, device="cuda")
    d_out = torch.empty_like(d_in)
    nbytes, bound = C.c_ulonglong(), C.c_double()
    err = C.create_string_buffer(512)
    s = torch.cuda.current_stream().cuda_stream
    # a zero bound is an argument error (std::invalid_argument)
    rc = lib.caller_round_trip_f32(d_in.data_ptr(), 32, 32, 32, 0.0, 0.0, d_cmp.data_ptr(), d_out.data_ptr(), s,
                                   C.byref(nbytes), C.byref(bound), err, 512)
    assert rc == 1 and err.value.startswith(b"invalid_argument"), err.value
    # a corrupt header is a codec error (std::runtime_error), and the context stays usable
    rc = lib.caller_round_trip_f32(d_in.data_ptr(), 32, 32, 32, 1e-3, 0.0, d_cmp.data_ptr(), d_out.data_ptr(), s,
                                   C.byref(nbytes), C.byref(bound), err, 512)
    assert rc == 0, err.value
    d_cmp[0] = 0xff
    rc = lib.caller_decode_f32(d_cmp.data_ptr(), 32, 32, 32, d_out.data_ptr(), s, err, 512)
    assert rc == 2 and err.value.startswith(b"runtime_error"), err.value
    torch.cuda.synchronize()


@pytest.mark.parametrize("nxyz,dtype,kind,rel,abs_bound", CASES[:3])
def test_decompress_length_from_header(nxyz, dtype, kind, rel, abs_bound):
    """waltz_b200_decompress(bytes = 0) reads the archive length from the
    header and decodes exactly like the call given the length, with trailing
    device bytes after the archive ignored."""
    import torch
    import waltz_b200
    from waltz_b200 import _lib
    a = _field(nxyz, dtype, kind)
    eb = rel * (float(a.max()) - float(a.min())) if rel else abs_bound
    archive = O.compress(a, eb)
    padded = torch.from_numpy(np.frombuffer(archive + b"\xa5" * 4096, np.uint8).copy()).cuda()
    out = torch.empty(a.shape, dtype=torch.float32 if dtype == np.float32 else torch.float64, device="cuda")
    nx, ny, nz = nxyz
    rc = _lib.lib().waltz_b200_decompress(C.c_void_p(padded.data_ptr()), 0, a.itemsize, nx, ny, nz,
                                          C.c_void_p(out.data_ptr()), out.numel() * a.itemsize,
                                          C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.last_error()
    assert out.cpu().numpy().tobytes() == O.decompress(archive, a.shape, dtype).tobytes()
    # the explicit length still rejects trailing data
    with pytest.raises(waltz_b200.WaltzError):
        _lib.checked(_lib.lib().waltz_b200_decompress(C.c_void_p(padded.data_ptr()), len(archive) + 8, a.itemsize,
                                                      nx, ny, nz, C.c_void_p(out.data_ptr()),
                                                      out.numel() * a.itemsize,
                                                      C.c_void_p(torch.cuda.current_stream().cuda_stream)))


def _filter():
    from tests.test_dropin import FILTER_FN, plugin
    lib = plugin()
    fn = FILTER_FN(C.cast(lib.H5PLget_plugin_info().contents.filter, C.c_void_p).value)
    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    libc.free.argtypes = [C.c_void_p]
    return fn, libc


def _run_filter(fn, libc, flags, cd, data: bytes):
    ptr = libc.malloc(len(data))
    C.memmove(ptr, data, len(data))
    buf, size = C.c_void_p(ptr), C.c_size_t(len(data))
    words = (C.c_uint * 6)(*cd)
    n = fn(flags, 6, words, len(data), C.byref(size), C.byref(buf))
    if n == 0:
        assert buf.value == ptr
        libc.free(ptr)
        return None
    out = C.string_at(buf.value, n)
    assert size.value == n
    libc.free(buf.value)
    return out


@pytest.mark.parametrize("nxyz,dtype,kind,rel,abs_bound", CASES[:3])
def test_h5z_filter_chunks_match_oracle(nxyz, dtype, kind, rel, abs_bound):
    from pywaltz.hdf5 import filter_values
    fn, libc = _filter()
    a = _field(nxyz, dtype, kind)
    eb = rel * (float(a.max()) - float(a.min())) if rel else abs_bound
    cd = filter_values(a.shape, dtype, eb)
    archive = _run_filter(fn, libc, 0, cd, a.tobytes())
    assert archive == O.compress(a, eb)
    back = _run_filter(fn, libc, 0x0100, cd, archive)
    assert back == O.decompress(archive, a.shape, dtype).tobytes()
    # a corrupt archive fails and leaves the buffer as it was
    assert _run_filter(fn, libc, 0x0100, cd, b"\xff" + archive[1:]) is None


def test_h5z_filter_reads_reference_cpu_chunks():
    if not O.ref_available():
        pytest.skip("reference CPU codec not built (oracle/Makefile ref)")
    from pywaltz.hdf5 import filter_values
    fn, libc = _filter()
    ref = O.RefCodec(O.AVX2)
    for nxyz, dtype in [((64, 64, 64), np.float32), ((40, 44, 52), np.float64)]:
        a = _field(nxyz, dtype, "grf", seed=5)
        eb = 1e-3 * (float(a.max()) - float(a.min()))
        archive = ref.compress(a, eb)
        back = _run_filter(fn, libc, 0x0100, filter_values(a.shape, dtype, eb), archive)
        assert back == ref.decompress(archive, a.shape, dtype).tobytes()


@pytest.mark.parametrize("nxyz,dtype,kind,rel,abs_bound", CASES[:3])
def test_pywaltz_shim_matches_oracle(nxyz, dtype, kind, rel, abs_bound):
    import pywaltz
    a = _field(nxyz, dtype, kind)
    eb = rel * (float(a.max()) - float(a.min())) if rel else abs_bound
    archive = pywaltz.compress(a, abs_error=eb)
    assert archive == O.compress(a, eb)
    out = pywaltz.decompress(archive, shape=a.shape, dtype=dtype)
    assert out.dtype == dtype and out.shape == a.shape
    assert out.tobytes() == O.decompress(archive, a.shape, dtype).tobytes()
    with pytest.raises(ValueError):
        pywaltz.decompress(b"\xff" + archive[1:], shape=a.shape, dtype=dtype)
