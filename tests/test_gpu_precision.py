"""GPU: the precision form's tensor-core splits.

Every split (TF32x3, BF16x3, exact bf16 slices) against the float64 matrix of
the lifting transform (from the oracle's plane-schedule transform of unit
columns), round trips of each form within the bound with the form recorded
in the header, the exact form's compression ratio against the plain form on
a double field with a sharp front, malformed split codes rejected, and the
batched decoder on archives of every form.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPLITS = {"matrix": 1, "matrix-bf16": 2, "matrix-exact": 3}
# the split code of each form, in the top two bits of header byte 3 (the z band)
BAND_CODE = {"matrix": 0, "matrix-bf16": 1, "matrix-exact": 2}


def _lib():
    from waltz_b200 import _lib
    return _lib.lib()


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _z_matrix_f64(nz: int, inverse: bool) -> np.ndarray:
    m = np.empty((nz, nz))
    for k in range(nz):
        e = np.zeros((nz, 1, 1))
        e[k] = 1.0
        m[:, k] = O.transform(e, inverse=False).reshape(nz)
    return np.linalg.inv(m) if inverse else m


# relative tolerance of the coefficient error against
# (max row sum of |M|) x (max |x|), per split and sample type
TOL = {("matrix", 4): 4e-6, ("matrix", 8): 4e-6, ("matrix-bf16", 4): 1e-6, ("matrix-bf16", 8): 1e-6,
       ("matrix-exact", 4): 1e-7, ("matrix-exact", 8): 1e-8}


@pytest.mark.parametrize("form", list(SPLITS))
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", [(64, 64, 64), (32, 24, 40), (16, 20, 33), (20, 20, 9), (24, 16, 65), (16, 16, 96),
                                  (20, 12, 128)])
def test_split_z_transform_matches_float64(nxyz, dtype, form):
    import torch
    nx, ny, nz = nxyz
    if form == "matrix-exact" and nz > 96:
        pytest.skip("the exact slices serve nz <= 96")
    rng = np.random.default_rng(nx * 7 + nz)
    a = rng.standard_normal((nz, ny, nx)) * np.exp(rng.uniform(-3, 3, (1, ny, nx)))  # columns of mixed scale
    a = a.astype(dtype)
    width = np.dtype(dtype).itemsize
    for inverse in (False, True):
        m = _z_matrix_f64(nz, inverse)
        expect = (m @ a.reshape(nz, -1).astype(np.float64)).reshape(a.shape)
        d = torch.from_numpy(a.copy()).cuda()
        rc = _lib().waltz_b200_zmatrix_split(C.c_void_p(d.data_ptr()), width, nx, ny, nz, int(inverse),
                                             SPLITS[form], _stream())
        assert rc == 0, _lib().waltz_b200_last_error()
        got = d.cpu().numpy().astype(np.float64)
        # per column: error against that column's row-weighted maximum
        colmax = np.abs(a.astype(np.float64)).reshape(nz, -1).max(axis=0)
        scale = np.abs(m).sum(axis=1).max() * colmax
        err = np.abs(got - expect).reshape(nz, -1).max(axis=0)
        worst = float((err / np.maximum(scale, 1e-300)).max())
        assert worst <= TOL[(form, width)], (inverse, worst)


def _front_field(shape, dtype=np.float64):
    from waltz_b200 import synthetic as S
    nz = shape[0]
    a = S.power_law_field(shape, 2, slope=-5.0 / 3.0, dtype=np.float64)
    a += 10.0 * np.tanh((np.arange(nz, dtype=np.float64) - nz / 2) / 2.0)[:, None, None]
    return a.astype(dtype)


def _spiky_field(shape):
    from waltz_b200 import synthetic as S
    a = S.power_law_field(shape, 3)
    rng = np.random.default_rng(3)
    spikes = rng.random(a.shape) < 0.01
    a[spikes] = np.where(rng.random(int(spikes.sum())) < 0.5, -50.0, 50.0)
    return a


@pytest.mark.parametrize("form", ["matrix-bf16", "matrix-exact"])
@pytest.mark.parametrize("shape,dtype,eb", [((64, 128, 128), np.float32, 1e-3), ((33, 24, 40), np.float32, 1e-5),
                                            ((96, 32, 48), np.float64, 1e-6), ((24, 64, 64), np.float64, 1e-4)])
def test_split_form_round_trip(form, shape, dtype, eb):
    """Each split form: header flag bit 6, the split code in the top bits of
    the z-band byte, the reference decoder (the oracle) rejects the archive,
    the GPU decoder restores every sample within the bound, twice
    identically."""
    import waltz_b200
    a = _spiky_field(shape) if dtype == np.float32 else _front_field(shape)
    if dtype == np.float32:
        eb = float(eb * (a.max() - a.min()))
    plain = waltz_b200.compress(a, abs_error=eb)
    arc = waltz_b200.compress(a, abs_error=eb, form=form)
    assert arc[0] == plain[0] | 0x40
    assert arc[3] == plain[3] | (BAND_CODE[form] << 6)
    with pytest.raises(Exception):
        O.decompress(arc, a.shape, dtype)
    out1 = waltz_b200.decompress(arc, shape=a.shape, dtype=dtype)
    out2 = waltz_b200.decompress(arc, shape=a.shape, dtype=dtype)
    assert out1.tobytes() == out2.tobytes()
    err = np.abs(out1.astype(np.longdouble) - a.astype(np.longdouble)).max()
    assert err <= np.longdouble(eb)


def test_exact_form_keeps_the_plain_ratio_on_double_fields():
    """Double field with a sharp front at ABS 1e-4 (the double configuration's
    bound, at 96 x 192 x 192): the exact slices move the compression
    ratio by well under 2 % against the plain form, where the fp32-accurate
    TF32x3 split loses several per cent to extra repairs."""
    import waltz_b200
    a = _front_field((96, 192, 192))  # plane schedule: 5 XY levels, 4 Z levels
    eb = 1e-4
    sizes = {f: len(waltz_b200.compress(a, abs_error=eb, form=f)) for f in ("plain", "matrix", "matrix-exact")}
    exact_change = sizes["plain"] / sizes["matrix-exact"] - 1.0
    assert abs(exact_change) <= 0.02, sizes
    arc = waltz_b200.compress(a, abs_error=eb, form="matrix-exact")
    out = waltz_b200.decompress(arc, shape=a.shape, dtype=np.float64)
    assert float(np.abs(out - a).max()) <= eb


def test_undefined_split_code_rejected():
    """Flag bits 5 and 7 are refused (bit 5 is the reference's CUDA fused
    plane-Z profile), band bits 6-7 mean nothing without flag bit 6, and the
    band code 3 is an undefined split: the decoder refuses each archive."""
    import waltz_b200
    a = _spiky_field((24, 64, 64))
    eb = float(1e-3 * (a.max() - a.min()))
    plain = bytearray(waltz_b200.compress(a, abs_error=eb))
    exact = bytearray(waltz_b200.compress(a, abs_error=eb, form="matrix-exact"))
    for arc, byte, flip in ((plain, 0, 0x20), (plain, 0, 0x80), (exact, 0, 0x20), (plain, 3, 0x40),
                            (exact, 3, 0xc0)):
        bad = bytearray(arc)
        bad[byte] |= flip
        with pytest.raises(waltz_b200.WaltzError):
            waltz_b200.decompress(bytes(bad), shape=a.shape, dtype=np.float32)
    # the exact form is refused above nz = 96, the other splits are not
    tall = _spiky_field((112, 32, 32))
    with pytest.raises(waltz_b200.WaltzError, match="matrix form"):
        waltz_b200.compress(tall, abs_error=eb, form="matrix-exact")
    assert len(waltz_b200.compress(tall, abs_error=eb, form="matrix-bf16")) > 32


def test_batched_decode_of_every_form():
    """One batched decode over archives of the plain form and every split
    equals the single decodes."""
    import torch
    import waltz_b200
    fields, forms = [], ["plain", "matrix", "matrix-bf16", "matrix-exact"]
    for k, form in enumerate(forms):
        a = _front_field((40 + 8 * k, 32, 48))  # plane schedule: 2 XY levels, 3 Z levels
        fields.append((a, form))
    archives = [waltz_b200.compress(a, abs_error=1e-5, form=f) for a, f in fields]
    dev = [torch.from_numpy(np.frombuffer(arc, np.uint8).copy()).cuda() for arc in archives]
    outs = waltz_b200.decompress_batch(dev, [a.shape for a, _ in fields], np.float64)
    for (a, _), arc, out in zip(fields, archives, outs):
        single = waltz_b200.decompress(arc, shape=a.shape, dtype=np.float64)
        assert out.cpu().numpy().tobytes() == single.tobytes()
