"""GPU parity against the reference's own CUDA library (src/waltz.cu and
src/lossless/wzp.cu of the reference, compiled for sm_100a by
``make -C oracle refgpu``): on the same device, inputs and bound, its archives
equal the product's byte for byte and each decoder reads the other's archives
bit-exactly. The CPU oracle stays the primary checker; this pins the product
to the reference GPU path as well (the reference's interop test,
cpu/tests/interop_gpu.cu:159-268, runs the same cross checks between its GPU
and CPU codecs)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from tests import patterns as P

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.refgpu_available(), reason="reference CUDA library not built")]

# the reference's Config drops unit dimensions, and its compressor takes 3-D
# fields only: every side at least 2
SHAPES = [s for s in P.CODEC_SHAPES if min(s) > 1] + [(40, 33, 21), (130, 9, 70)]


def _torch():
    import torch
    return torch


def _ref_compress(field, eb):
    torch = _torch()
    lib = O.refgpu_lib()
    cap = lib.refgpu_capacity(field.numel(), field.element_size())
    out = torch.empty(cap, dtype=torch.uint8, device=field.device)
    src = field.clone()  # the reference takes a mutable input pointer
    size = O.refgpu_compress(src.data_ptr(), field.element_size(), tuple(field.shape), eb, out.data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out[:size]


def _ref_decompress(archive, shape, dtype):
    torch = _torch()
    out = torch.empty(shape, dtype=dtype, device=archive.device)
    O.refgpu_decompress(archive.data_ptr(), out.element_size(), tuple(shape), out.data_ptr(),
                        torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out


def _check(field, eb):
    import waltz_b200
    torch = _torch()
    ours = waltz_b200.compress_tensor(field, eb)
    theirs = _ref_compress(field, eb)
    assert ours.numel() == theirs.numel() and torch.equal(ours, theirs)
    mine = waltz_b200.decompress_tensor(ours, tuple(field.shape), field.dtype)
    assert torch.equal(_ref_decompress(ours, tuple(field.shape), field.dtype), mine)
    assert torch.equal(waltz_b200.decompress_tensor(theirs, tuple(field.shape), field.dtype), mine)
    assert float((mine.double() - field.double()).abs().max()) <= eb


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nxyz", SHAPES)
def test_same_archive_as_reference_gpu(nxyz, dtype):
    torch = _torch()
    for pattern in (2, 3, 4, 5):
        a = P.codec_field(P.zyx(nxyz), pattern, 1e-3, dtype)
        _check(torch.from_numpy(a).cuda(), 1e-3)


@pytest.mark.parametrize("shape,dtype", [((128, 128, 128), "f32"), ((64, 256, 256), "f32"),
                                         ((96, 256, 384), "f64"), ((33, 200, 72), "f32")])
@pytest.mark.parametrize("rel", [1e-3, 1e-5])
def test_same_archive_as_reference_gpu_synthetic(shape, dtype, rel):
    import waltz_b200
    from waltz_b200.synthetic import power_law_field_device
    torch = _torch()
    f = power_law_field_device(shape, 7, dtype=torch.float32 if dtype == "f32" else torch.float64).contiguous()
    _check(f, waltz_b200.rel_to_abs_bound(f, rel))
