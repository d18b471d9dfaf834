"""GPU parity: the CUDA library, called through its C ABI, against the C
oracle (bit/byte-exact) on the reference's own test shapes and patterns."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests import patterns as P

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _lib():
    from waltz_b200 import _lib
    return _lib.lib()


def _stream():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


def gpu_transform(a: np.ndarray, inverse: bool) -> np.ndarray:
    torch = _torch()
    d = torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()
    nz, ny, nx = a.shape
    rc = _lib().waltz_b200_transform(C.c_void_p(d.data_ptr()), a.itemsize, nx, ny, nz, int(inverse), _stream())
    assert rc == 0, _lib().waltz_b200_last_error()
    return d.cpu().numpy()


def gpu_compress(a: np.ndarray, eb: float) -> bytes:
    import waltz_b200
    return waltz_b200.compress(a, abs_error=eb)


def gpu_decompress(archive: bytes, shape, dtype) -> np.ndarray:
    import waltz_b200
    return waltz_b200.decompress(archive, shape=shape, dtype=dtype)


TRANSFORM_SHAPES = P.CODEC_SHAPES + [(96, 40, 24), (130, 9, 70), (40, 44, 52), (100, 3, 33), (31, 64, 8),
                                     (64, 65, 66), (200, 17, 9)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", TRANSFORM_SHAPES)
def test_transform_bit_exact(nxyz, dtype):
    rng = np.random.default_rng(sum(nxyz) + 7)
    a = rng.standard_normal(P.zyx(nxyz)).astype(dtype)
    f = gpu_transform(a, inverse=False)
    assert f.tobytes() == O.transform(a, inverse=False).tobytes()
    i = gpu_transform(f, inverse=True)
    assert i.tobytes() == O.transform(f, inverse=True).tobytes()


def test_wzp_encode_byte_exact():
    torch = _torch()
    for n, pattern, mag, sign in P.wzp_cases():
        if n == 0:
            continue
        expect = O.wzp_encode(mag, sign)
        dm = torch.from_numpy(mag.astype(np.int16).view(np.int16)).cuda()
        ds = torch.from_numpy(sign.view(np.int32)).cuda()
        cap = O.oracle_lib().wo_wzp_max_bytes(n)
        out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        written = C.c_size_t()
        rc = _lib().waltz_b200_wzp_encode(C.c_void_p(dm.data_ptr()), C.c_void_p(ds.data_ptr()), n,
                                          C.c_void_p(out.data_ptr()), cap, C.byref(written), _stream())
        assert rc == 0, _lib().waltz_b200_last_error()
        got = out[:written.value].cpu().numpy().tobytes()
        assert got == expect, (n, pattern)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", P.CODEC_SHAPES)
def test_archive_byte_exact_and_decode_bit_exact(nxyz, dtype):
    for pattern in range(5):
        a = P.codec_field(P.zyx(nxyz), pattern, 1e-3, dtype)
        expect = O.compress(a, 1e-3)
        got = gpu_compress(a, 1e-3)
        assert got == expect, pattern
        out = gpu_decompress(got, a.shape, dtype)
        assert out.tobytes() == O.decompress(expect, a.shape, dtype).tobytes()
        err = np.abs(out.astype(np.longdouble) - a.astype(np.longdouble)).max()
        assert err <= np.longdouble(1e-3)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_side_channels_byte_exact(dtype):
    cases = [((17, 19, 23), 5, 1e-5), ((9, 11, 17), 6, 1e-5), ((17, 19, 23), 2, 1e-7), ((64, 64, 64), 1, 1e-5),
             ((23, 19, 17), 2, 1e-12)]
    import waltz_b200
    for nxyz, pattern, eb in cases:
        a = P.codec_field(P.zyx(nxyz), pattern, eb, dtype)
        try:
            expect = O.compress(a, eb)
        except O.CodecError:
            with pytest.raises(waltz_b200.WaltzError):
                gpu_compress(a, eb)
            continue
        got = gpu_compress(a, eb)
        assert got == expect, (nxyz, pattern, eb)
        assert gpu_decompress(got, a.shape, dtype).tobytes() == O.decompress(expect, a.shape, dtype).tobytes()


def test_golden_fixtures_on_gpu():
    from tests.golden import load_golden
    import hashlib
    for case in load_golden():
        field = case["input"]
        got = gpu_compress(field, case["abs_error"])
        assert got == case["archive"], case["name"]
        out = gpu_decompress(got, field.shape, field.dtype)
        assert hashlib.sha256(out.tobytes()).hexdigest() == case["decoded_sha256"], case["name"]


@pytest.mark.parametrize("case", ["powerlaw_f32", "front_f64_plane", "spiky_f32_plane"])
def test_larger_fields_byte_exact(case):
    from waltz_b200 import synthetic as S
    if case == "powerlaw_f32":
        a = S.power_law_field((96, 128, 160), 1)
        eb = S.rel_to_abs(a, 1e-4)
    elif case == "front_f64_plane":
        a = S.front_field((48, 128, 96), 2)
        eb = 1e-6
    else:
        a = S.spiky_field((40, 128, 128), 3)
        eb = S.rel_to_abs(a, 1e-5)
    expect = O.compress(a, eb)
    got = gpu_compress(a, eb)
    assert got == expect
    out = gpu_decompress(got, a.shape, a.dtype)
    assert out.tobytes() == O.decompress(expect, a.shape, a.dtype).tobytes()


def test_invalid_inputs_rejected():
    import waltz_b200
    a = P.codec_field((17, 11, 9), 2, 1e-3, np.float32)
    for bad in (np.nan, np.inf, -np.inf):
        b = a.copy()
        b.reshape(-1)[7] = bad
        with pytest.raises(waltz_b200.WaltzError):
            gpu_compress(b, 1e-3)
    for eb in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(ValueError):
            gpu_compress(a, eb)


def test_malformed_archives_rejected():
    import waltz_b200
    from tests.test_oracle import _mutations
    a = P.codec_field((23, 19, 17), 3, 1e-5, np.float64)
    archive = O.compress(a, 1e-5)
    for bad in _mutations(archive, a.size):
        with pytest.raises((waltz_b200.WaltzError, ValueError)):
            gpu_decompress(bad, a.shape, np.float64)
    # the untouched archive still decodes after all the rejections
    assert gpu_decompress(archive, a.shape, np.float64).tobytes() == O.decompress(archive, a.shape, np.float64).tobytes()


def test_unordered_side_records_accepted_duplicates_rejected():
    """cpu/tests/test_codec.cpp:288-301: swapped side records decode to the same
    bits; a duplicated index is rejected."""
    import struct
    import waltz_b200
    a = P.codec_field((23, 19, 17), 3, 1e-5, np.float64)
    archive = bytearray(O.compress(a, 1e-5))
    expected = O.decompress(bytes(archive), a.shape, np.float64)
    wzp = struct.unpack_from("<Q", archive, 16)[0]
    np_ = struct.unpack_from("<I", archive, 24)[0]
    assert np_ >= 2
    pi = 32 + ((wzp + 7) & ~7)
    pv = pi + ((np_ * 4 + 7) & ~7)
    swapped = bytearray(archive)
    for start, width in ((pi, 4), (pv, 8)):
        first = bytes(swapped[start:start + width])
        last = bytes(swapped[start + (np_ - 1) * width:start + np_ * width])
        swapped[start:start + width] = last
        swapped[start + (np_ - 1) * width:start + np_ * width] = first
    out = gpu_decompress(bytes(swapped), a.shape, np.float64)
    assert out.tobytes() == expected.tobytes()
    dup = bytearray(swapped)
    dup[pi + 4:pi + 8] = dup[pi:pi + 4]
    with pytest.raises(waltz_b200.WaltzError):
        gpu_decompress(bytes(dup), a.shape, np.float64)


def test_extrema():
    import waltz_b200
    torch = _torch()
    for dtype in (torch.float32, torch.float64):
        t = torch.randn(3, 1000, 77, dtype=dtype, device="cuda") * 5
        lo, hi = waltz_b200.extrema(t)
        assert lo == float(t.min()) and hi == float(t.max())


def test_decode_chunk_canonical():
    torch = _torch()
    nx, ny, nz = 33, 31, 17
    a = P.codec_field(P.zyx((nx, ny, nz)), 2, 1e-3, np.float32)
    archive = O.compress(a, 1e-3)
    src = torch.from_numpy(np.frombuffer(archive, np.uint8).copy()).cuda()
    out = torch.empty(a.shape, dtype=torch.float32, device="cuda")
    err = _lib().waltz_cuda_decode_chunk(nx, ny, nz, 4, C.c_void_p(src.data_ptr()), len(archive),
                                         C.c_void_p(out.data_ptr()), out.numel() * 4, _stream())
    assert err is None, err
    assert out.cpu().numpy().tobytes() == O.decompress(archive, a.shape, np.float32).tobytes()
    # wrong geometry / width / length are rejected with a diagnostic
    assert _lib().waltz_cuda_decode_chunk(nx, ny, 8, 4, C.c_void_p(src.data_ptr()), len(archive),
                                          C.c_void_p(out.data_ptr()), nx * ny * 8 * 4, _stream()) is not None
    wide = torch.empty(a.shape, dtype=torch.float64, device="cuda")
    assert _lib().waltz_cuda_decode_chunk(nx, ny, nz, 8, C.c_void_p(src.data_ptr()), len(archive),
                                          C.c_void_p(wide.data_ptr()), wide.numel() * 8, _stream()) is not None
    assert _lib().waltz_cuda_decode_chunk(nx, ny, nz, 4, C.c_void_p(src.data_ptr()), len(archive) - 8,
                                          C.c_void_p(out.data_ptr()), out.numel() * 4, _stream()) is not None


def test_lookback_wait_is_bounded():
    """A chunk that never publishes its lookback state makes its successor's
    bounded wait expire: the call fails with a diagnostic, without a hang."""
    torch = _torch()
    from waltz_b200 import synthetic as S
    a = S.power_law_field((64, 64, 64), 5)
    d = torch.from_numpy(a).cuda()
    cap = _lib().waltz_b200_compressed_capacity(a.size, 4)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    rc = _lib().waltz_b200_test_lookback_timeout(C.c_void_p(d.data_ptr()), 4, 64, 64, 64, 1e-3,
                                                 C.c_void_p(out.data_ptr()), cap, 3, 2000, _stream())
    assert rc != 0
    assert b"lookback" in _lib().waltz_b200_last_error()
    # the context stays usable
    assert gpu_compress(a, 1e-3) == O.compress(a, 1e-3)


def test_batch_decode_matches_oracle():
    """waltz_gpu_decode_batch: clipped edge tiles, two sides, a missing tile
    (fill), against per-tile oracle decodes."""
    torch = _torch()
    from waltz_b200 import loader
    from waltz_b200 import synthetic as S
    tile, frame, samples = (16, 24, 20), (30, 40, 33), 2
    fields = [[S.power_law_field(frame, 10 + 2 * s + side) for side in range(2)] for s in range(samples)]
    batch_samples, expect = [], np.zeros((2, samples, *frame), np.float32)
    for s in range(samples):
        sample = []
        for side in range(2):
            blobs = loader.frame_to_archives(fields[s][side], tile, 1e-3, O.compress)
            if s == 1 and side == 0:
                blobs[1] = None  # missing tile -> fill
            sample.append(blobs)
            for k, origin in enumerate(loader.tile_origins(frame, tile)):
                region = tuple(slice(o, min(o + t, n)) for o, t, n in zip(origin, tile, frame))
                if blobs[k] is None:
                    expect[(side, s, *region)] = -7.0
                    continue
                dec = O.decompress(blobs[k], tile, np.float32)
                expect[(side, s, *region)] = dec[tuple(slice(0, r.stop - r.start) for r in region)]
        batch_samples.append(sample)
    batch = loader.pack(batch_samples, indexed=True)
    out = loader.decode_batch(batch, tile=tile, frame=frame, width=4, sides=2, fill=-7.0)
    torch.cuda.synchronize()
    assert out.cpu().numpy().tobytes() == expect.tobytes()


def _z_matrix_f64(nz: int, inverse: bool) -> np.ndarray:
    """The all-levels Z analysis of a column as a matrix, from the oracle's
    float64 plane-schedule transform of unit columns (nx = ny = 1)."""
    m = np.empty((nz, nz))
    for k in range(nz):
        e = np.zeros((nz, 1, 1))
        e[k] = 1.0
        m[:, k] = O.transform(e, inverse=False).reshape(nz)
    return np.linalg.inv(m) if inverse else m


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", [(64, 64, 64), (32, 24, 40), (16, 20, 33), (256, 4, 17), (20, 20, 9), (24, 16, 65),
                                  (16, 16, 96), (20, 12, 128)])
def test_tensor_core_z_transform_matches_float64(nxyz, dtype):
    """The precision form's tensor-core Z transform (TF32 hi/lo halves, FP32
    accumulation; a double field rounded to float first) against the float64
    matrix of the lifting transform, for columns of up to 128 samples (two
    MMA passes of 64 planes above 64); the coefficient error is a few 2^-20
    of the row-weighted input."""
    torch = _torch()
    nx, ny, nz = nxyz
    rng = np.random.default_rng(nx * 7 + nz)
    a = rng.standard_normal((nz, ny, nx)).astype(dtype)
    entry = _lib().waltz_b200_zmatrix if dtype == np.float32 else _lib().waltz_b200_zmatrix_f64
    for inverse in (False, True):
        m = _z_matrix_f64(nz, inverse)
        expect = (m @ a.reshape(nz, -1).astype(np.float64)).reshape(a.shape)
        d = torch.from_numpy(a.copy()).cuda()
        rc = entry(C.c_void_p(d.data_ptr()), nx, ny, nz, int(inverse), _stream())
        assert rc == 0, _lib().waltz_b200_last_error()
        got = d.cpu().numpy().astype(np.float64)
        scale = np.abs(m).sum(axis=1).max() * np.abs(a).max()
        err = np.abs(got - expect).max()
        assert err <= 4e-6 * scale, (inverse, err, scale)


@pytest.mark.parametrize("rel", [1e-3, 1e-5])
@pytest.mark.parametrize("shape", [(64, 128, 128), (24, 96, 64), (33, 24, 40), (96, 64, 96), (128, 32, 64)])
def test_matrix_form_round_trip(shape, rel):
    """Precision form (tensor-core Z stage): the archive carries header bit 6,
    the reference decoder (the oracle) rejects it, the GPU decoder restores
    every sample within the bound, twice identically, and the archive stays
    close to the plain form's size. The field: k^-11/3 random field with 1 %
    salt spikes of magnitude 50, the shape of the tensor-core configuration."""
    import waltz_b200
    from waltz_b200 import synthetic as S
    a = S.power_law_field(shape, 3)
    rng = np.random.default_rng(3)
    spikes = rng.random(a.shape) < 0.01
    a[spikes] = np.where(rng.random(int(spikes.sum())) < 0.5, -50.0, 50.0)
    eb = float(rel * (a.max() - a.min()))
    plain = waltz_b200.compress(a, abs_error=eb)
    matrix = waltz_b200.compress(a, abs_error=eb, form="matrix")
    assert matrix[0] == plain[0] | 0x40
    with pytest.raises(Exception):
        O.decompress(matrix, a.shape, np.float32)
    out1 = waltz_b200.decompress(matrix, shape=a.shape, dtype=np.float32)
    out2 = waltz_b200.decompress(matrix, shape=a.shape, dtype=np.float32)
    assert out1.tobytes() == out2.tobytes()
    err = np.abs(out1.astype(np.longdouble) - a.astype(np.longdouble)).max()
    assert err <= np.longdouble(eb)
    assert abs(len(matrix) - len(plain)) <= 0.05 * len(plain) + 256


def test_matrix_form_rejects_unsuited_fields():
    import waltz_b200
    cube = np.zeros((64, 64, 64), np.float32)  # dyadic schedule: no separate Z stage
    with pytest.raises(waltz_b200.WaltzError, match="matrix form"):
        waltz_b200.compress(cube, abs_error=1e-3, form="matrix")
    with pytest.raises(waltz_b200.WaltzError, match="matrix form"):
        waltz_b200.compress(np.zeros((160, 64, 64), np.float32), abs_error=1e-3, form="matrix")  # nz > 128
    big = np.zeros((24, 64, 64))
    big[5, 6, 7] = 1e39  # a double the float transform cannot hold
    with pytest.raises(waltz_b200.WaltzError, match="float range"):
        waltz_b200.compress(big, abs_error=1e-3, form="matrix")
    assert len(waltz_b200.compress(big, abs_error=1e30)) > 32  # the plain form takes it


@pytest.mark.parametrize("shape,eb", [((96, 32, 48), 1e-6), ((24, 64, 64), 1e-4), ((128, 16, 24), 1e-8)])
def test_matrix_form_round_trip_float64(shape, eb):
    """Precision form of a double field (the configuration with nz = 96 in
    small): fp32-accurate tensor-core Z stage, quantisation and repair
    decisions in double; every sample within the bound, decodes repeatable,
    header bit 6 set. The field: k^-5/3 random field plus a tanh front along
    z, in double."""
    import waltz_b200
    from waltz_b200 import synthetic as S
    nz, ny, nx = shape
    a = S.power_law_field(shape, 2, slope=-5.0 / 3.0, dtype=np.float64)
    a += 10.0 * np.tanh((np.arange(nz, dtype=np.float64) - nz / 2) / 2.0)[:, None, None]
    plain = waltz_b200.compress(a, abs_error=eb)
    matrix = waltz_b200.compress(a, abs_error=eb, form="matrix")
    assert matrix[0] == plain[0] | 0x40
    out1 = waltz_b200.decompress(matrix, shape=a.shape, dtype=np.float64)
    out2 = waltz_b200.decompress(matrix, shape=a.shape, dtype=np.float64)
    assert out1.tobytes() == out2.tobytes()
    err = np.abs(out1.astype(np.longdouble) - a.astype(np.longdouble)).max()
    assert err <= np.longdouble(eb)


BATCH_FORMS = [(0, 1), (0, 3), (1, 32), (2, 1), (2, 4)]  # (stage-batched | field chains | work queue, width)


@pytest.fixture(params=BATCH_FORMS, ids=lambda f: f"mode{f[0]}w{f[1]}")
def batch_form(request):
    lib = _lib()
    assert lib.waltz_b200_batch_config(*request.param) == 0
    yield request.param
    lib.waltz_b200_batch_config(1, 32)


def test_batch_compress_equals_single_calls(batch_form):
    """Batched compress of uneven chunks (one CUDA graph): every archive is
    byte-identical to the single-call archive of its chunk, on the first call
    and on the replay, and a few archives equal the oracle's directly;
    per-chunk bounds differ."""
    torch = _torch()
    import waltz_b200
    from waltz_b200 import synthetic as S
    rng = np.random.default_rng(4)
    sides = [16, 17, 32, 48, 64]
    fields, bounds, hosts = [], [], []
    for k in range(14):
        shape = tuple(int(rng.choice(sides)) for _ in range(3))
        a = S.power_law_field(shape, 40 + k) * float(10 ** rng.uniform(-2, 3))
        hosts.append(a)
        fields.append(torch.from_numpy(a).cuda())
        bounds.append(1e-3 * float(a.max() - a.min()))
    out = torch.empty(sum(waltz_b200.compressed_capacity(f.numel(), 4) + 16 for f in fields), dtype=torch.uint8,
                      device="cuda")
    for _ in range(2):
        archives = waltz_b200.compress_batch(fields, bounds, out=out)
        for f, eb, arc in zip(fields, bounds, archives):
            single = waltz_b200.compress_tensor(f, eb)
            assert torch.equal(arc, single)
    for a, eb, arc in list(zip(hosts, bounds, archives))[::5]:
        assert arc.cpu().numpy().tobytes() == O.compress(a, eb)
    # a failing item is reported with its index
    bad = fields[:3] + [torch.full((8, 8, 8), float("nan"), device="cuda")]
    with pytest.raises(waltz_b200.WaltzError, match="batch item 3"):
        waltz_b200.compress_batch(bad, 1e-3)


def _uneven_batch(torch, seed, count, sides=(16, 17, 32, 48, 64)):
    from waltz_b200 import synthetic as S
    rng = np.random.default_rng(seed)
    fields, bounds = [], []
    for k in range(count):
        shape = tuple(int(rng.choice(sides)) for _ in range(3))
        a = S.power_law_field(shape, seed * 100 + k) * float(10 ** rng.uniform(-2, 3))
        fields.append(torch.from_numpy(a).cuda())
        bounds.append(1e-3 * float(a.max() - a.min()))
    return fields, bounds


def test_batch_decompress_equals_single_calls(batch_form):
    """Batched decode of uneven archives of both forms into one preallocated
    tensor: bit-identical to the single-call decode; a second batch of other
    archives with the same shapes replays the graph; host header copies and a
    list of output tensors give the same result."""
    torch = _torch()
    import waltz_b200
    from waltz_b200 import synthetic as S
    fields, bounds = _uneven_batch(torch, 5, 12)
    # three precision-form archives (plane schedule, nz <= 128; the last in
    # two MMA passes of up to 64 planes)
    for shape in [(24, 96, 64), (33, 24, 40), (96, 32, 48)]:
        fields.append(torch.from_numpy(S.power_law_field(shape, 9)).cuda())
        bounds.append(1e-3)
    forms = ["plain"] * 12 + ["matrix"] * 3
    shapes = [tuple(f.shape) for f in fields]
    total = sum(f.numel() for f in fields)
    out = torch.full((total,), float("nan"), dtype=torch.float32, device="cuda")
    for rnd in range(2):
        if rnd:  # other archives, same shapes and forms: the graph is replayed
            fields = [f * 1.5 + 0.25 for f in fields]
        archives = [waltz_b200.compress_tensor(f, eb, form=fm) for f, eb, fm in zip(fields, bounds, forms)]
        # archives in one staging buffer, like a loader's packed upload
        staging = torch.cat(archives)
        views, at = [], 0
        for a in archives:
            views.append(staging[at:at + a.numel()])
            at += a.numel()
        got = waltz_b200.decompress_batch(views, shapes, torch.float32, out=out)
        for a, s, g, f, eb in zip(archives, shapes, got, fields, bounds):
            single = waltz_b200.decompress_tensor(a, s, torch.float32)
            assert torch.equal(g, single)
            assert float((g.double() - f.double()).abs().max()) <= eb
    hdrs = [bytes(a[:32].cpu().numpy()) for a in archives]
    outs = [torch.empty(s, dtype=torch.float32, device="cuda") for s in shapes]
    got = waltz_b200.decompress_batch(archives, shapes, torch.float32, out=outs, headers=hdrs)
    for a, s, g in zip(archives, shapes, got):
        assert torch.equal(g, waltz_b200.decompress_tensor(a, s, torch.float32))


def test_batch_decompress_f64_and_errors(batch_form):
    torch = _torch()
    import waltz_b200
    from waltz_b200 import synthetic as S
    fields = [torch.from_numpy(S.power_law_field(s, 11).astype(np.float64)).cuda()
              for s in [(16, 16, 16), (20, 33, 18), (40, 24, 32), (96, 32, 48)]]
    # the last in the precision form (a double field, nz = 96)
    archives = [waltz_b200.compress_tensor(f, 1e-6, form="matrix" if k == 3 else "plain")
                for k, f in enumerate(fields)]
    shapes = [tuple(f.shape) for f in fields]
    got = waltz_b200.decompress_batch(archives, shapes, torch.float64)
    for a, s, g in zip(archives, shapes, got):
        assert torch.equal(g, waltz_b200.decompress_tensor(a, s, torch.float64))
    # a truncated archive is reported with its index
    bad = archives[:2] + [archives[2][:-8]] + archives[3:]
    with pytest.raises(waltz_b200.WaltzError, match="batch item 2"):
        waltz_b200.decompress_batch(bad, shapes, torch.float64)
    # a shape that does not match the archive's levels
    with pytest.raises(waltz_b200.WaltzError, match="batch item 1"):
        waltz_b200.decompress_batch(archives, [shapes[0], (64, 64, 64)] + shapes[2:], torch.float64)


def test_batch_config_rejects_invalid_forms():
    lib = _lib()
    assert lib.waltz_b200_batch_config(3, 4) == -1
    assert lib.waltz_b200_batch_config(0, 0) == -1
    assert lib.waltz_b200_batch_config(1, 65) == -1
    assert b"invalid batch configuration" in lib.waltz_b200_last_error()
    assert lib.waltz_b200_batch_config(1, 32) == 0


def test_tuning_knobs_never_change_the_bytes():
    """Every knob value of the tuning table gives the same archives and the
    same decoded samples (single fields of both schedules and both dtypes,
    and a batch in every execution form)."""
    torch = _torch()
    import waltz_b200
    from waltz_b200 import autotune as A
    from waltz_b200 import synthetic as S
    lib = _lib()
    cases = [((40, 72, 96), np.float32), ((24, 96, 64), np.float32), ((33, 40, 48), np.float64),
             ((20, 200, 136), np.float32), ((96, 96, 96), np.float32), ((64, 80, 48), np.float64)]
    try:
        for shape, dt in cases:
            f = torch.from_numpy(S.power_law_field(shape, 3).astype(dt)).cuda()
            ref = waltz_b200.compress_tensor(f, 1e-3, tuned=False)
            dref = waltz_b200.decompress_tensor(ref, shape, f.dtype, tuned=False)
            extra = [{"small_inv": 0, "small_fwd": 0}, {"small_inv": 1 << 30, "small_fwd": 1 << 30},
                     {"xy_march": 1}, {"xy_march": 2}, {"xy_march": 3, "stage_kernels": 0},
                     {"xy_march": 3, "small_inv": 0}, {"small_march": 1 << 21}, {"small_march": 1 << 30},
                     {"small_march_fwd": 1 << 21}, {"small_march_fwd": 1 << 30, "small_march": 1 << 30}]
            for k in A.SINGLE_CANDIDATES + extra:
                A.set_single(lib, k)
                arc = waltz_b200.compress_tensor(f, 1e-3, tuned=False)
                assert torch.equal(arc, ref), (shape, k)
                assert torch.equal(waltz_b200.decompress_tensor(arc, shape, f.dtype, tuned=False), dref), (shape, k)
        A.set_single(lib, {})
        fields, bounds = _uneven_batch(torch, 8, 10)
        ref = [waltz_b200.compress_tensor(f, eb, tuned=False) for f, eb in zip(fields, bounds)]
        for k in A.BATCH_CANDIDATES:
            assert lib.waltz_b200_batch_config(k["mode"], k["width"]) == 0
            A.set_single(lib, A.batch_single_knobs(k))
            arcs = waltz_b200.compress_batch(fields, bounds, tuned=False)
            assert all(torch.equal(a, r) for a, r in zip(arcs, ref)), k
            dec = waltz_b200.decompress_batch(arcs, [tuple(f.shape) for f in fields], torch.float32, tuned=False)
            for d, r, f in zip(dec, ref, fields):
                assert torch.equal(d, waltz_b200.decompress_tensor(r, tuple(f.shape), torch.float32, tuned=False))
        assert lib.waltz_b200_set_option(99, 1) == -1
        assert lib.waltz_b200_set_option(A.OPT_ZMARCH_PLANES, -1) == -1
    finally:
        A.set_single(lib, {})
        lib.waltz_b200_batch_config(1, 32)


def test_unaligned_archive_addresses():
    """Archives written to and decoded from odd device addresses give the same
    bytes and samples (the side-record sections then take byte-wide paths)."""
    torch = _torch()
    import waltz_b200
    from waltz_b200 import _lib as L
    from waltz_b200 import synthetic as S
    lib = _lib()
    for shape, dt in [((48, 64, 80), np.float32), ((20, 33, 40), np.float64)]:
        f = torch.from_numpy(S.power_law_field(shape, 21).astype(dt)).cuda()
        ref = waltz_b200.compress_tensor(f, 1e-4)  # many repair records at this bound
        assert int.from_bytes(bytes(ref[24:28].cpu().numpy()), "little") > 0
        nz, ny, nx = shape
        w = f.element_size()
        cap = waltz_b200.compressed_capacity(f.numel(), w)
        buf = torch.zeros(cap + 16, dtype=torch.uint8, device="cuda")
        written = C.c_size_t()
        for off in (1, 3):
            L.checked(lib.waltz_b200_compress(C.c_void_p(f.data_ptr()), w, nx, ny, nz, 1e-4,
                                              C.c_void_p(buf.data_ptr() + off), cap, C.byref(written), _stream()))
            assert torch.equal(buf[off:off + written.value], ref)
            out = torch.empty_like(f)
            L.checked(lib.waltz_b200_decompress(C.c_void_p(buf.data_ptr() + off), written.value, w, nx, ny, nz,
                                                C.c_void_p(out.data_ptr()), out.numel() * w, _stream()))
            assert torch.equal(out, waltz_b200.decompress_tensor(ref, shape, f.dtype))


@pytest.mark.parametrize("small_march", [1 << 15, 1 << 40])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", [(64, 64, 64), (37, 41, 50), (96, 80, 72), (130, 129, 128)])
def test_dyadic_small_levels_as_marches_match_oracle(nxyz, dtype, small_march):
    """Dyadic fields whose small levels (every level, with the largest
    threshold, the finest one's repair and final emitters included) run as
    marches: the inverse as a Z march then an XY march instead of the tile
    inverse, the forward as an XY march then a Z march instead of the
    z-march. Transforms, archives and decodes equal the oracle's."""
    import torch
    import waltz_b200
    from waltz_b200 import autotune as A
    from waltz_b200 import synthetic as S
    lib = _lib()
    rng = np.random.default_rng(sum(nxyz) + 9)
    a = rng.standard_normal(P.zyx(nxyz)).astype(dtype)
    g = S.power_law_field(P.zyx(nxyz), 8).astype(dtype)
    eb = 1e-4 * (float(g.max()) - float(g.min()))
    assert lib.waltz_b200_set_option(A.OPT_SMALL_MARCH, small_march) == 0
    assert lib.waltz_b200_set_option(A.OPT_SMALL_MARCH_FWD, small_march) == 0
    try:
        f = gpu_transform(a, inverse=False)
        assert f.tobytes() == O.transform(a, inverse=False).tobytes()
        assert gpu_transform(f, inverse=True).tobytes() == O.transform(f, inverse=True).tobytes()
        d = torch.from_numpy(g).cuda()
        arc = waltz_b200.compress_tensor(d, eb, tuned=False)
        host = arc.cpu().numpy().tobytes()
        assert host == O.compress(g, eb)
        out = waltz_b200.decompress_tensor(arc, g.shape, dtype, tuned=False).cpu().numpy()
        assert out.tobytes() == O.decompress(host, g.shape, dtype).tobytes()
    finally:
        lib.waltz_b200_set_option(A.OPT_SMALL_MARCH, 0)
        lib.waltz_b200_set_option(A.OPT_SMALL_MARCH_FWD, 0)


@pytest.mark.parametrize("xy_march", [0, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", [(64, 40, 100), (200, 17, 9), (9, 11, 65), (48, 32, 9), (33, 31, 130),
                                  (72, 80, 24), (40, 36, 257)])
def test_plane_schedule_per_level_z_matches_oracle(nxyz, dtype, xy_march):
    """Plane-schedule fields with the whole-stage kernels off: every Z level
    runs as the per-column register march (forward and inverse, ragged last
    windows, reflection at both ends), and the XY levels as the staged
    kernels or, with the knob, the warp march (X across lanes); transforms,
    archives and decodes equal the oracle's."""
    import torch
    import waltz_b200
    from waltz_b200 import autotune as A
    from waltz_b200 import synthetic as S
    lib = _lib()
    rng = np.random.default_rng(sum(nxyz) + 5)
    a = rng.standard_normal(P.zyx(nxyz)).astype(dtype)
    g = S.power_law_field(P.zyx(nxyz), 7).astype(dtype)
    eb = 1e-4 * (float(g.max()) - float(g.min()))
    assert lib.waltz_b200_set_option(A.OPT_STAGE_KERNELS, 0) == 0
    assert lib.waltz_b200_set_option(A.OPT_XY_MARCH, xy_march) == 0
    try:
        f = gpu_transform(a, inverse=False)
        assert f.tobytes() == O.transform(a, inverse=False).tobytes()
        assert gpu_transform(f, inverse=True).tobytes() == O.transform(f, inverse=True).tobytes()
        d = torch.from_numpy(g).cuda()
        arc = waltz_b200.compress_tensor(d, eb, tuned=False)  # untuned: the knob stays off
        host = arc.cpu().numpy().tobytes()
        assert host == O.compress(g, eb)
        out = waltz_b200.decompress_tensor(arc, g.shape, dtype, tuned=False).cpu().numpy()
        assert out.tobytes() == O.decompress(host, g.shape, dtype).tobytes()
    finally:
        lib.waltz_b200_set_option(A.OPT_STAGE_KERNELS, 1)
        lib.waltz_b200_set_option(A.OPT_XY_MARCH, 0)
