"""Batched GPU decode for training loops: the device side of the reference's
WaltzGPUDataLoader (python/pywaltz/gpu_dataloader.py:126-236) on this
library's ``waltz_gpu_decode_batch``.

Wire format (python/pywaltz/_raw_chunks.py:391-409): archive blobs, each
starting on a 16-byte boundary, then a 16-byte-aligned table of little-endian
(u64 offset, u64 size) pairs in sample / side / (z, y, x) tile order; size 0
marks a missing tile that is filled with `fill`.
"""
from __future__ import annotations

import ctypes as C
import math
import struct
from dataclasses import dataclass
from itertools import product

import numpy as np

from ._lib import BatchShape, WaltzError, lib


@dataclass
class WireBatch:
    payload: "object"  # torch uint8 tensor (CPU, optionally pinned)
    spans: list
    count: int
    indexed: bool = False

    def pin_memory(self):
        return WireBatch(self.payload.pin_memory(), self.spans, self.count, self.indexed)


def pack(samples, *, indexed=True):
    """samples: list of samples; a sample is a list of frames (1 or 2 sides);
    a frame is a list of archive bytes (or None) per tile."""
    import torch
    data, spans = bytearray(), []
    for sample in samples:
        for frame in sample:
            for blob in frame:
                if blob is None:
                    spans.append((0, 0))
                else:
                    data.extend(b"\0" * (-len(data) % 16))
                    spans.append((len(data), len(blob)))
                    data.extend(blob)
    if indexed:
        data.extend(b"\0" * (-len(data) % 16))
        entry = struct.Struct("<QQ")
        for offset, size in spans:
            data.extend(entry.pack(offset, size))
    payload = torch.frombuffer(bytearray(data), dtype=torch.uint8) if data else torch.empty(0, dtype=torch.uint8)
    return WireBatch(payload, spans, len(samples), indexed)


def tile_origins(frame_shape, tile):
    """Tile origins of a (z, y, x) or (y, x) frame in the wire order."""
    return product(*(range(0, n, c) for n, c in zip(frame_shape, tile)))


def scratch_bytes(tile, jobs, width, bz=16):
    stride = (math.prod(tile) + 3) & ~3
    return 3 * stride * jobs * width + 8 * 256 * 32 * 4 + 16


def decode_batch(batch: WireBatch, *, tile, frame, width, sides=1, fill=0.0, out=None, scratch=None,
                 device="cuda", stream=None):
    """Decode every tile of a packed batch into one (sides, samples, *frame)
    CUDA tensor with a single library call on the current stream."""
    import torch
    if not batch.indexed:
        raise ValueError("the batch must carry its span table (indexed=True)")
    tile3 = (*reversed(tuple(tile)), 1, 1)[:3]
    frame3 = (*reversed(tuple(frame)), 1, 1)[:3]
    shape = BatchShape(*tile3, *frame3, batch.count, sides, width)
    jobs = len(batch.spans)
    dtype = torch.float32 if width == 4 else torch.float64
    if out is None:
        out = torch.empty((sides, batch.count, *frame), dtype=dtype, device=device)
    if scratch is None:
        scratch = torch.empty(scratch_bytes(tile, jobs, width), dtype=torch.uint8, device=device)
    host = batch.payload
    packed = host.to(device, non_blocking=True)
    s = stream if stream is not None else torch.cuda.current_stream()
    err = lib().waltz_gpu_decode_batch(C.byref(shape), C.c_void_p(host.data_ptr()), C.c_void_p(packed.data_ptr()),
                                       packed.numel(), C.c_void_p(scratch.data_ptr()), scratch.numel(),
                                       C.c_void_p(out.data_ptr()), out.numel() * width, float(fill),
                                       C.c_void_p(s.cuda_stream))
    if err is not None:
        raise WaltzError(f"Waltz batch decode: {err.decode(errors='replace')}")
    return out


def frame_to_archives(field: np.ndarray, tile, abs_error, compress):
    """Split a (z, y, x) field into tiles (edge tiles zero-padded to the tile
    shape, as an HDF5 chunked dataset stores them) and compress each."""
    blobs = []
    for origin in tile_origins(field.shape, tile):
        region = tuple(slice(o, o + t) for o, t in zip(origin, tile))
        block = np.zeros(tile, field.dtype)
        part = field[region]
        block[tuple(slice(0, s) for s in part.shape)] = part
        blobs.append(compress(block, abs_error))
    return blobs
