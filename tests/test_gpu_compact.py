"""GPU: compact repair sections (the reference's opt-in WPW1 profile).

* With WALTZ_B200_OPT_COMPACT_REPAIRS = 16 or 64 the archive equals the
  oracle's compact form of the plain archive byte for byte (groups of 32 in
  order); the GPU decode equals the oracle's and the reference CPU codec's
  decode of it bit for bit, within the bound.
* Archives the reference CUDA library writes in this profile
  (WALTZ_SMALL_PWE_SCALE=16, unordered records, groups placed by an atomic
  counter) decode here exactly as the reference's own decoders decode them.
* Malformed compact sections are refused here and by the reference CPU
  decoder alike (never handed to the reference CUDA decoder, which traps on
  them).
* The C++ API takes the reference's WALTZ_SMALL_PWE_SCALE switch.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import patterns as P

pytestmark = pytest.mark.gpu

OPT_COMPACT = 5


def _lib():
    from waltz_b200 import _lib
    return _lib.lib()


def _field(nxyz, dtype, kind, seed=5):
    from waltz_b200 import synthetic as S
    zyx = P.zyx(nxyz)
    if kind == "sin":
        return S.sinusoids(zyx, seed=seed, dtype=dtype)
    return S.power_law_field(zyx, seed, dtype=dtype)


def _compress_compact(a, eb, scale):
    import waltz_b200
    lib = _lib()
    assert lib.waltz_b200_set_option(OPT_COMPACT, scale) == 0
    try:
        return waltz_b200.compress(a, abs_error=eb)
    finally:
        lib.waltz_b200_set_option(OPT_COMPACT, 0)


CASES = [((64, 64, 64), np.float32, "sin", 1e-3), ((64, 64, 64), np.float32, "grf", 1e-5),
         ((40, 44, 52), np.float64, "grf", 1e-4), ((96, 40, 24), np.float32, "grf", 1e-4),
         ((48, 32, 96), np.float64, "grf", 1e-6), ((33, 24, 40), np.float32, "grf", 1e-5)]


@pytest.mark.parametrize("scale", [16, 64])
@pytest.mark.parametrize("nxyz,dtype,kind,rel", CASES)
def test_compact_archive_matches_oracle(nxyz, dtype, kind, rel, scale):
    import waltz_b200
    a = _field(nxyz, dtype, kind)
    eb = rel * (float(a.max()) - float(a.min()))
    arc = _compress_compact(a, eb, scale)
    plain = O.compress(a, eb)
    expect = O.compact_repairs(plain, a, eb / scale)
    assert arc == expect
    np_ = int.from_bytes(plain[24:28], "little")
    if np_ >= 32:
        assert arc[0] & 2, "a field with repairs packs its section"
        assert len(arc) < len(plain)
    out = waltz_b200.decompress(arc, shape=a.shape, dtype=dtype)
    assert out.tobytes() == O.decompress(arc, a.shape, dtype).tobytes()
    if O.ref_available():
        assert out.tobytes() == O.RefCodec(O.AVX2).decompress(arc, a.shape, dtype).tobytes()
    assert float(np.abs(out.astype(np.float64) - a.astype(np.float64)).max()) <= eb
    # the default profile is untouched by the option once it is reset
    assert waltz_b200.compress(a, abs_error=eb) == plain


@pytest.mark.parametrize("nxyz,dtype", [((64, 64, 64), np.float32), ((40, 44, 52), np.float64),
                                        ((48, 32, 96), np.float64)])
def test_reference_gpu_compact_archives_decode_identically(nxyz, dtype):
    """The reference CUDA library's own compact archives (dyadic float and
    double fields, and a double plane field: none of them takes its fused
    plane-Z profile) decode here as the reference CUDA and CPU decoders
    decode them."""
    if not O.refgpu_available():
        pytest.skip("reference CUDA library not built")
    import torch
    import waltz_b200
    a = _field(nxyz, dtype, "grf", seed=9)
    eb = 1e-4 * (float(a.max()) - float(a.min()))
    d = torch.from_numpy(a.copy()).cuda()
    lib = O.refgpu_lib()
    cap = lib.refgpu_capacity(d.numel(), d.element_size())
    arch = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    os.environ["WALTZ_SMALL_PWE_SCALE"] = "16"
    try:
        size = O.refgpu_compress(d.data_ptr(), d.element_size(), a.shape, eb, arch.data_ptr(), s)
    finally:
        del os.environ["WALTZ_SMALL_PWE_SCALE"]
    torch.cuda.synchronize()
    arc = arch[:size].cpu().numpy().tobytes()
    assert arc[0] & 2 and not arc[0] & 0x20, "a compact archive of the lifting profile"
    ours = waltz_b200.decompress(arc, shape=a.shape, dtype=dtype)
    if O.ref_available():
        assert ours.tobytes() == O.RefCodec(O.AVX2).decompress(arc, a.shape, dtype).tobytes()
    ref_out = torch.empty_like(d)
    O.refgpu_decompress(arch.data_ptr(), d.element_size(), a.shape, ref_out.data_ptr(), s)
    torch.cuda.synchronize()
    assert ours.tobytes() == ref_out.cpu().numpy().tobytes()
    assert float(np.abs(ours.astype(np.float64) - a.astype(np.float64)).max()) <= eb


def test_malformed_compact_sections_refused():
    import waltz_b200
    a = _field((64, 64, 64), np.float32, "grf")
    eb = 1e-5 * (float(a.max()) - float(a.min()))
    arc = bytearray(_compress_compact(a, eb, 16))
    assert arc[0] & 2
    wb = int.from_bytes(arc[16:24], "little")
    np_ = int.from_bytes(arc[24:28], "little")
    pi = 32 + (wb + 7) // 8 * 8
    pv = pi + (np_ * 4 + 7) // 8 * 8
    groups = (np_ + 31) // 32
    bad_cases = {
        "magic": (pv, b"XPW1"),
        "groups": (pv + 4, (groups + 1).to_bytes(4, "little")),
        "payload bytes": (pv + 8, (1 << 40).to_bytes(8, "little")),
        "step": (pv + 16, np.float64(-1.0).tobytes()),
        "misaligned group": (pv + 24, (4).to_bytes(4, "little")),
        "group beyond payload": (pv + 24, (0x7ffffff8).to_bytes(4, "little")),
    }
    last = np_ - (groups - 1) * 32
    if last < 32:  # a mask bit past the last group's records
        bad_cases["mask"] = (pv + 24 + 8 * (groups - 1) + 4, (1 << last).to_bytes(4, "little"))
    for what, (at, raw) in bad_cases.items():
        bad = bytearray(arc)
        bad[at:at + len(raw)] = raw
        with pytest.raises(waltz_b200.WaltzError):
            waltz_b200.decompress(bytes(bad), shape=a.shape, dtype=np.float32)
        with pytest.raises(O.CodecError):
            O.decompress(bytes(bad), a.shape, np.float32)
        if O.ref_available():
            with pytest.raises(O.CodecError):
                O.RefCodec(O.AVX2).decompress(bytes(bad), a.shape, np.float32)
    # the section must be smaller than the native errors it replaces
    native_size = bytearray(arc)
    native_size[4:8] = (np_ * 4).to_bytes(4, "little")
    with pytest.raises(waltz_b200.WaltzError):
        waltz_b200.decompress(bytes(native_size), shape=a.shape, dtype=np.float32)


def test_cxx_api_takes_the_reference_switch():
    """WALTZ::d_compress with WALTZ_SMALL_PWE_SCALE=64 writes the compact
    profile (as the reference's d_compress does); the variable unset, the
    default profile."""
    import torch
    from tests.test_gpu_dropin import _caller
    lib = _caller("ours")
    a = _field((64, 64, 64), np.float32, "grf")
    eb = 1e-5 * (float(a.max()) - float(a.min()))
    d_in = torch.from_numpy(a).cuda()
    from waltz_b200 import compressed_capacity
    d_cmp = torch.zeros(compressed_capacity(a.size, 4), dtype=torch.uint8, device="cuda")
    d_out = torch.empty_like(d_in)
    nbytes, bound = C.c_ulonglong(), C.c_double()
    err = C.create_string_buffer(512)
    s = torch.cuda.current_stream().cuda_stream
    os.environ["WALTZ_SMALL_PWE_SCALE"] = "64"
    try:
        rc = lib.caller_round_trip_f32(d_in.data_ptr(), 64, 64, 64, 0.0, eb, d_cmp.data_ptr(), d_out.data_ptr(), s,
                                       C.byref(nbytes), C.byref(bound), err, 512)
    finally:
        del os.environ["WALTZ_SMALL_PWE_SCALE"]
    assert rc == 0, err.value
    arc = d_cmp[:nbytes.value].cpu().numpy().tobytes()
    assert arc == O.compact_repairs(O.compress(a, eb), a, eb / 64)
    assert d_out.cpu().numpy().tobytes() == O.decompress(arc, a.shape, np.float32).tobytes()
    os.environ["WALTZ_SMALL_PWE_SCALE"] = "7"
    try:
        rc = lib.caller_round_trip_f32(d_in.data_ptr(), 64, 64, 64, 0.0, eb, d_cmp.data_ptr(), d_out.data_ptr(), s,
                                       C.byref(nbytes), C.byref(bound), err, 512)
    finally:
        del os.environ["WALTZ_SMALL_PWE_SCALE"]
    assert rc == 1 and b"WALTZ_SMALL_PWE_SCALE" in err.value
