"""The chunk-container GPU data loader end to end: frames of uneven chunks
decoded by the batched graph into fresh tensors, equal to per-chunk decodes
assembled on the host side, graph replay across batches, serial mode."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _frames(torch, count, frame, seed):
    from waltz_b200.synthetic import power_law_field_device
    return [power_law_field_device(frame, seed + i) * (1 + i) for i in range(count)]


def _expected(torch, path, i):
    """Frame i assembled from per-chunk single-call decodes."""
    import waltz_b200
    from waltz_b200 import loader as L
    ds = L.ChunkedFrames(path)
    out = torch.full(ds.shape, ds.fill, dtype=torch.float32, device="cuda")
    for o, s, blob in ds[i][0]:
        arc = torch.frombuffer(bytearray(blob), dtype=torch.uint8).cuda()
        out[o[0]:o[0] + s[0], o[1]:o[1] + s[1], o[2]:o[2] + s[2]] = waltz_b200.decompress_tensor(arc, s, torch.float32)
    return out


def test_loader_uneven_chunks_fill_and_lead(tmp_path):
    import torch
    from waltz_b200 import loader as L
    frame = (40, 70, 90)
    frames = _frames(torch, 5, frame, 30)
    eb = 1e-3
    path = tmp_path / "frames.wzc"
    L.write_frames(path, frames, L.tiles(frame, (32, 32, 64)), eb, fill=-7.0, skip={(3, 2)})
    dl = L.WaltzGPUDataLoader(path, batch_size=2, lead=1)
    seen = 0
    for inp, tgt in dl:
        for k in range(inp.shape[0]):
            i = seen + k
            assert torch.equal(inp[k], _expected(torch, path, i))
            assert torch.equal(tgt[k], _expected(torch, path, i + 1))
        seen += inp.shape[0]
    assert seen == 4
    # bound against the original, the skipped chunk reads as the fill value
    ds = L.ChunkedFrames(path)
    got = next(iter(L.WaltzGPUDataLoader(path, batch_size=5)))
    for i in range(5):
        mask = torch.ones(frame, dtype=torch.bool, device="cuda")
        if i == 3:
            (o, s) = L.tiles(frame, (32, 32, 64))[2]
            mask[o[0]:o[0] + s[0], o[1]:o[1] + s[1], o[2]:o[2] + s[2]] = False
            assert bool((got[i][~mask] == -7.0).all())
        assert float((got[i][mask].double() - frames[i][mask].double()).abs().max()) <= eb
    assert len(ds) == 5


def test_loader_replays_one_graph_and_matches_serial(tmp_path):
    import torch
    from waltz_b200 import _lib
    from waltz_b200 import loader as L
    frame = (24, 48, 80)
    frames = _frames(torch, 6, frame, 50)
    path = tmp_path / "frames.wzc"
    L.write_frames(path, frames, L.tiles(frame, (16, 32, 48)), 1e-3)
    lib = _lib.lib()
    before = lib.waltz_b200_graph_count()
    batched = [b.clone() for b in L.WaltzGPUDataLoader(path, batch_size=2)]
    assert lib.waltz_b200_graph_count() - before == 1  # three batches, one capture
    serial = list(L.WaltzGPUDataLoader(path, batch_size=2, decode_mode="serial"))
    assert len(batched) == len(serial) == 3
    for a, b in zip(batched, serial):
        assert torch.equal(a, b)


def test_loader_with_a_worker_process(tmp_path):
    import torch
    from waltz_b200 import loader as L
    frame = (16, 40, 64)
    frames = _frames(torch, 3, frame, 70)
    path = tmp_path / "frames.wzc"
    L.write_frames(path, frames, L.tiles(frame, (16, 16, 32)), 1e-3)
    got = list(L.WaltzGPUDataLoader(path, batch_size=3, num_workers=1))
    assert len(got) == 1
    for i in range(3):
        assert torch.equal(got[0][i], _expected(torch, path, i))
