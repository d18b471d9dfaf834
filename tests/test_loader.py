"""Host side of the chunk-container data loader (no GPU): container index,
packing of a batch on 16-byte boundaries, box validation."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from waltz_b200 import loader as L


def _container(path, frame, samples, fill=-1.0, width=4):
    """A container with random 'archives' (opaque bytes) per chunk box."""
    rng = np.random.default_rng(7)
    blobs, index = [], []
    at = L._HEADER.size
    at += -at % 16
    for boxes in samples:
        entries = []
        for o, s in boxes:
            blob = rng.integers(0, 256, int(rng.integers(32, 300)), dtype=np.uint8).tobytes()
            entries.append((o, s, at, blob))
            at += len(blob)
            at += -at % 16
        index.append(entries)
    idx = bytearray()
    for entries in index:
        idx += struct.pack("<I", len(entries))
        for o, s, off, blob in entries:
            idx += L._CHUNK.pack(*o, *s, off, len(blob))
    with open(path, "wb") as fh:
        fh.write(L._HEADER.pack(L.MAGIC, width, *frame, len(samples), fill, at, len(idx)))
        pos = L._HEADER.size
        for entries in index:
            for o, s, off, blob in entries:
                fh.write(b"\0" * (off - pos))
                fh.write(blob)
                pos = off + len(blob)
        fh.write(b"\0" * (at - pos))
        fh.write(idx)
    return index


def test_tiles_cover_the_frame_once():
    frame = (40, 70, 90)
    boxes = L.tiles(frame, (32, 32, 64))
    cover = np.zeros(frame, np.int32)
    for o, s in boxes:
        cover[o[0]:o[0] + s[0], o[1]:o[1] + s[1], o[2]:o[2] + s[2]] += 1
    assert (cover == 1).all()
    assert len({s for _, s in boxes}) > 1  # uneven edge chunks


def test_container_index_and_packing(tmp_path):
    frame = (20, 33, 40)
    boxes = L.tiles(frame, (16, 16, 32))
    index = _container(tmp_path / "f.wzc", frame, [boxes, boxes[:-2], boxes], fill=-1.5)
    ds = L.ChunkedFrames(tmp_path / "f.wzc", lead=1)
    assert ds.shape == frame and ds.width == 4 and ds.fill == -1.5 and len(ds) == 2
    item = ds[1]  # frames 1 and 2
    assert len(item) == 2
    for frame_records, entries in zip(item, (index[1], index[2])):
        assert [(o, s) for o, s, _ in frame_records] == [(o, s) for o, s, _, _ in entries]
        assert [b for _, _, b in frame_records] == [b for _, _, _, b in entries]
    batch = L.pack_chunks([ds[0], ds[1]])
    assert batch.count == 2
    payload = batch.payload.numpy().tobytes()
    for side, i, o, s, off, size in batch.chunks:
        assert off % 16 == 0
        rec = ds[i][side]
        blob = next(b for oo, ss, b in rec if oo == o and ss == s)
        assert payload[off:off + size] == blob
    with pytest.raises(IndexError):
        ds[2]


def test_container_rejects_bad_boxes(tmp_path):
    frame = (16, 16, 16)
    _container(tmp_path / "a.wzc", frame, [[((0, 0, 0), (16, 16, 16)), ((8, 0, 0), (8, 8, 8))]])
    with pytest.raises(ValueError, match="overlap"):
        L.ChunkedFrames(tmp_path / "a.wzc")
    _container(tmp_path / "b.wzc", frame, [[((0, 0, 8), (16, 16, 16))]])
    with pytest.raises(ValueError, match="outside"):
        L.ChunkedFrames(tmp_path / "b.wzc")
    (tmp_path / "c.wzc").write_bytes(b"nope" + bytes(60))
    with pytest.raises(ValueError, match="container"):
        L.ChunkedFrames(tmp_path / "c.wzc")
