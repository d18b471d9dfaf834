"""Pins the C oracle restatement (oracle/waltz_oracle.c) against the
reference CPU codec compiled from its own sources (oracle/_ref) and against
the committed golden fixtures. CPU only."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import oracle as O
from tests import patterns as P

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference CPU codec not built (make -C oracle ref)")


def test_levels_and_zband():
    for n in [1, 2, 8, 9, 16, 17, 33, 64, 100, 257, 512, 1000, 100000]:
        expected, length = 0, n
        while length > 8 and expected < 5:
            length -= length // 2
            expected += 1
        assert O.levels(n) == expected
    assert O.zband(512, 512, 512, 5, True) == 16
    assert O.zband(192, 192, 192, 5, True) == 6
    assert O.zband(32, 32, 3, 0, True) == 3
    assert O.zband(384, 256, 96, 4, False) == 2


@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", P.CODEC_SHAPES + [(96, 40, 24), (130, 9, 70)])
def test_transform_matches_reference(nxyz, dtype):
    rng = np.random.default_rng(sum(nxyz))
    a = rng.standard_normal(P.zyx(nxyz)).astype(dtype)
    f1, f2 = O.transform(a, inverse=False), O.ref_transform(a, inverse=False)
    assert f1.tobytes() == f2.tobytes()
    i1, i2 = O.transform(f1, inverse=True), O.ref_transform(f1, inverse=True)
    assert i1.tobytes() == i2.tobytes()
    # the reference's AVX2 tiles agree too (its own scalar/SIMD pin)
    assert O.ref_transform(f1, inverse=True, avx2=True).tobytes() == i2.tobytes()


@needs_ref
def test_wzp_matches_reference():
    for n, pattern, mag, sign in P.wzp_cases():
        if n == 0:
            continue
        s1, s2 = O.wzp_encode(mag, sign), O.ref_wzp_encode(mag, sign)
        assert s1 == s2, (n, pattern)
        m, s = O.wzp_decode(s1, n)
        assert np.array_equal(m, mag)
        nz = mag != 0
        bits = ((sign[np.arange(n) // 32] >> (np.arange(n) % 32)) & 1).astype(bool)
        got = ((s[np.arange(n) // 32] >> (np.arange(n) % 32)) & 1).astype(bool)
        assert np.array_equal(got, bits & nz), (n, pattern)


@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", P.CODEC_SHAPES)
def test_codec_matches_reference(nxyz, dtype):
    ref = O.RefCodec(O.SCALAR)
    for pattern in range(5):
        a = P.codec_field(P.zyx(nxyz), pattern, 1e-3, dtype)
        c1, c2 = O.compress(a, 1e-3), ref.compress(a, 1e-3)
        assert c1 == c2, pattern
        d1, d2 = O.decompress(c1, a.shape, dtype), ref.decompress(c2, a.shape, dtype)
        assert d1.tobytes() == d2.tobytes()
        err = np.abs(d1.astype(np.longdouble) - a.astype(np.longdouble)).max()
        assert err <= np.longdouble(1e-3)


@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_codec_side_channels_match_reference(dtype):
    ref = O.RefCodec(O.SCALAR)
    cases = [((17, 19, 23), 5, 1e-5), ((9, 11, 17), 6, 1e-5), ((17, 19, 23), 2, 1e-7), ((64, 64, 64), 1, 1e-5)]
    for nxyz, pattern, eb in cases:
        a = P.codec_field(P.zyx(nxyz), pattern, eb, dtype)
        try:
            c2 = ref.compress(a, eb)
        except O.CodecError:
            with pytest.raises(O.CodecError):
                O.compress(a, eb)
            continue
        c1 = O.compress(a, eb)
        assert c1 == c2
        assert O.decompress(c1, a.shape, dtype).tobytes() == ref.decompress(c2, a.shape, dtype).tobytes()


@needs_ref
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tight_bound_fails_closed_like_reference(dtype):
    a = P.codec_field((23, 19, 17), 2, 1e-12, dtype)
    ref = O.RefCodec(O.SCALAR)
    try:
        c2 = ref.compress(a, 1e-12)
    except O.CodecError:
        with pytest.raises(O.CodecError):
            O.compress(a, 1e-12)
        return
    assert O.compress(a, 1e-12) == c2


@needs_ref
def test_invalid_inputs_rejected_like_reference():
    ref = O.RefCodec(O.SCALAR)
    a = P.codec_field((17, 11, 9), 2, 1e-3, np.float32)
    for bad in (np.nan, np.inf, -np.inf):
        b = a.copy()
        b.reshape(-1)[7] = bad
        with pytest.raises(O.CodecError):
            O.compress(b, 1e-3)
        with pytest.raises(O.CodecError):
            ref.compress(b, 1e-3)
    for eb in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(O.CodecError):
            O.compress(a, eb)


def _mutations(archive: bytes, n: int):
    """Header mutations of cpu/tests/test_codec.cpp:256-270 plus truncations."""
    muts = [(0, 1, 0), (0, 1, 0x57), (0, 1, 24), (0, 1, 0x3C), (0, 1, 12), (1, 1, 255), (2, 1, 255),
            (3, 1, 0), (3, 1, 33), (4, 4, 0xFFFFFFFF), (16, 8, 2**64 - 1), (16, 8, 0), (24, 4, n + 1),
            (28, 4, n + 1)]
    for off, width, value in muts:
        b = bytearray(archive)
        b[off:off + width] = int(value).to_bytes(width, "little")
        yield bytes(b)
    for q in (0.0, -1.0, float("nan"), float("inf")):
        b = bytearray(archive)
        b[8:16] = np.float64(q).tobytes()
        yield bytes(b)
    for cut in (0, 1, 31, 32, 33, len(archive) // 2, len(archive) - 1):
        yield archive[:cut]


@needs_ref
def test_malformed_archives_rejected_like_reference():
    ref = O.RefCodec(O.SCALAR)
    a = P.codec_field((23, 19, 17), 3, 1e-5, np.float64)
    archive = O.compress(a, 1e-5)
    for bad in _mutations(archive, a.size):
        with pytest.raises(O.CodecError):
            O.decompress(bad, a.shape, np.float64)
        with pytest.raises(O.CodecError):
            ref.decompress(bad, a.shape, np.float64)


def test_golden_fixtures():
    """Archives produced by the reference CPU codec (tests/golden/make_golden.py)."""
    from tests.golden import load_golden
    cases = load_golden()
    assert cases, "golden fixtures missing"
    for case in cases:
        field = case["input"]
        archive = O.compress(field, case["abs_error"])
        assert archive == case["archive"], case["name"]
        out = O.decompress(archive, field.shape, field.dtype)
        assert hashlib.sha256(out.tobytes()).hexdigest() == case["decoded_sha256"], case["name"]


@pytest.mark.parametrize("scale", [16, 64])
@pytest.mark.parametrize("nxyz,dtype,rel", [((40, 44, 52), np.float32, 1e-3), ((33, 24, 40), np.float64, 1e-5),
                                            ((64, 64, 64), np.float32, 1e-5)])
def test_oracle_compact_repairs_decode_like_the_reference(nxyz, dtype, rel, scale):
    """The oracle's compact (WPW1) repair sections decode bit for bit like the
    reference CPU codec decodes them, within the bound (cpu/src/codec.cpp:
    305-325 reads the section; src/small_pwe.cuh:21-94 defines it)."""
    if not O.ref_available():
        pytest.skip("reference CPU codec not built")
    from waltz_b200 import synthetic as S
    a = S.power_law_field(P.zyx(nxyz), 7, dtype=dtype)
    eb = rel * (float(a.max()) - float(a.min()))
    plain = O.compress(a, eb)
    arc = O.compact_repairs(plain, a, eb / scale)
    assert arc[0] & 2 and len(arc) < len(plain)
    ours = O.decompress(arc, a.shape, dtype)
    assert ours.tobytes() == O.RefCodec(O.SCALAR).decompress(arc, a.shape, dtype).tobytes()
    assert float(np.abs(ours.astype(np.float64) - a.astype(np.float64)).max()) <= eb
    bad = bytearray(arc)
    bad[4:8] = (len(plain)).to_bytes(4, "little")  # section length inconsistent with the layout
    with pytest.raises(O.CodecError):
        O.decompress(bytes(bad), a.shape, dtype)
