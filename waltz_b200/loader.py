"""Batched GPU decode for training loops: the device side of the reference's
WaltzGPUDataLoader (python/pywaltz/gpu_dataloader.py:23-181).

Two paths:
 * the reference's own wire format (python/pywaltz/_raw_chunks.py:107-125):
   archive blobs, each starting on a 16-byte boundary, then a 16-byte-aligned
   table of little-endian (u64 offset, u64 size) pairs in sample / side /
   (z, y, x) tile order; size 0 marks a missing tile that is filled with
   `fill`. One tile shape per batch; decoded by ``waltz_gpu_decode_batch``
   (`pack`, `decode_batch`).
 * frames stored as chunk archives of any shapes in a container file
   (`write_frames`, `ChunkedFrames`, `WaltzGPUDataLoader`): worker processes
   only read archive bytes and pack them into one pinned tensor per batch;
   the training process uploads it on a copy stream (overlapping the previous
   batch's decode) and decodes every chunk of the batch with one call of
   ``waltz_b200_decompress_batch`` straight into a fresh (batch, z, y, x)
   tensor, each chunk into its box of its frame. The decode graph is captured
   once per batch description (chunk shapes and places) and replayed for
   every later batch with the same description. New against the reference:
   a frame's chunks may have any shapes, and both transform forms decode. The
   reference reads its chunks from HDF5 files (filter 61197); the container
   below needs no HDF5 stack.

Container (little endian):
    header  b"WZC1", u32 width (4|8), u32 fz, fy, fx (frame), u64 samples,
            f64 fill, u64 index offset, u64 index bytes         (52 bytes)
    blobs   archives, each starting on a 16-byte boundary
    index   per sample: u32 chunk count, then per chunk
            u32 oz, oy, ox, u32 cz, cy, cx, u64 offset, u64 size
A frame region that no chunk covers holds `fill`.
"""

from __future__ import annotations

import ctypes as C
import math
import mmap
import os
import struct
from dataclasses import dataclass
from itertools import product

import numpy as np

from ._lib import Archive, BatchShape, WaltzError, checked, lib


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


# ------------------------------------------------------ uneven chunk frames
MAGIC = b"WZC1"
_HEADER = struct.Struct("<4sIIIIQdQQ")
_CHUNK = struct.Struct("<IIIIIIQQ")


def tiles(frame, tile):
    """Boxes (origin, shape) of a regular tiling of `frame` by `tile` with
    smaller edge boxes, both (z, y, x)."""
    out = []
    for oz in range(0, frame[0], tile[0]):
        for oy in range(0, frame[1], tile[1]):
            for ox in range(0, frame[2], tile[2]):
                o = (oz, oy, ox)
                out.append((o, tuple(min(t, f - a) for t, f, a in zip(tile, frame, o))))
    return out


def _check_boxes(boxes, frame):
    """Chunk boxes must lie inside the frame and not overlap."""
    if not boxes:
        return
    o = np.array([b[0] for b in boxes], dtype=np.int64)
    e = o + np.array([b[1] for b in boxes], dtype=np.int64)
    if (o < 0).any() or (e > np.array(frame)).any() or (e <= o).any():
        raise ValueError("a chunk box lies outside its frame")
    inter = (np.minimum(e[:, None], e[None]) > np.maximum(o[:, None], o[None])).all(-1)
    np.fill_diagonal(inter, False)
    if inter.any():
        raise ValueError("chunk boxes of a frame overlap")


def write_frames(path, frames, boxes, abs_error, *, fill=0.0, form="plain", skip=()):
    """Compress every frame (a (z,y,x) CUDA tensor, all of one shape and
    dtype) chunk by chunk on the GPU and write the container. `boxes` lists
    (origin, shape) per chunk, shared by all frames, or a callable giving the
    list for frame i; `skip` holds (frame, chunk) pairs to leave out (they
    read back as `fill`)."""
    import torch
    from . import compress_tensor
    frames = list(frames)
    if not frames:
        raise ValueError("no frames")
    shape, dtype = tuple(frames[0].shape), frames[0].dtype
    if len(shape) != 3 or dtype not in (torch.float32, torch.float64):
        raise ValueError("frames must be (z,y,x) float32/float64 tensors")
    width = 4 if dtype == torch.float32 else 8
    skip = set(skip)
    blobs, index = [], []
    at = _HEADER.size
    at += -at % 16
    for i, f in enumerate(frames):
        if tuple(f.shape) != shape or f.dtype != dtype:
            raise ValueError("frames differ in shape or dtype")
        entries = []
        fb = list(boxes(i) if callable(boxes) else boxes)
        _check_boxes(fb, shape)
        for k, (o, s) in enumerate(fb):
            if (i, k) in skip:
                continue
            region = f[o[0]:o[0] + s[0], o[1]:o[1] + s[1], o[2]:o[2] + s[2]].contiguous()
            blob = compress_tensor(region, abs_error, form=form).cpu().numpy().tobytes()
            entries.append((o, s, at, len(blob)))
            blobs.append((at, blob))
            at += len(blob)
            at += -at % 16
        index.append(entries)
    idx = bytearray()
    for entries in index:
        idx += struct.pack("<I", len(entries))
        for o, s, off, size in entries:
            idx += _CHUNK.pack(*o, *s, off, size)
    with open(path, "wb") as fh:
        fh.write(_HEADER.pack(MAGIC, width, *shape, len(frames), float(fill), at, len(idx)))
        pos = _HEADER.size
        for off, blob in blobs:
            fh.write(b"\0" * (off - pos))
            fh.write(blob)
            pos = off + len(blob)
        fh.write(b"\0" * (at - pos))
        fh.write(idx)


class ChunkedFrames:
    """Map-style dataset over a container file: item i is the list of raw
    chunk records (origin, shape, archive bytes) of frame i, and of frame
    i + lead as well when `lead` > 0. No decoding and no CUDA in workers."""

    def __init__(self, path, lead=0):
        self.path = os.fspath(path)
        self.lead = int(lead)
        with open(self.path, "rb") as fh:
            head = fh.read(_HEADER.size)
            if len(head) < _HEADER.size:
                raise ValueError("not a Waltz chunk container")
            magic, self.width, fz, fy, fx, samples, self.fill, io, il = _HEADER.unpack(head)
            if magic != MAGIC or self.width not in (4, 8):
                raise ValueError("not a Waltz chunk container")
            fh.seek(io)
            raw = fh.read(il)
        if len(raw) != il:
            raise ValueError("truncated container index")
        self.shape = (fz, fy, fx)
        self.samples = samples
        self.index, at = [], 0
        for _ in range(samples):
            (count,) = struct.unpack_from("<I", raw, at)
            at += 4
            entries = []
            for _ in range(count):
                oz, oy, ox, cz, cy, cx, off, size = _CHUNK.unpack_from(raw, at)
                at += _CHUNK.size
                if off % 16 or off + size > io or size < 32:
                    raise ValueError("invalid chunk record in the container index")
                entries.append(((oz, oy, ox), (cz, cy, cx), off, size))
            self.index.append(entries)
        if not 0 <= self.lead < max(1, samples):
            raise ValueError("lead must be in [0, number of samples)")
        for entries in self.index:
            _check_boxes([(o, s) for o, s, _, _ in entries], self.shape)
        self._map = None

    def __len__(self):
        return self.samples - self.lead

    def _bytes(self):
        if self._map is None:
            with open(self.path, "rb") as fh:
                self._map = mmap.mmap(fh.fileno(), 0, access=mmap.ACCESS_READ)
        return self._map

    def _frame(self, i):
        m = self._bytes()
        return [(o, s, bytes(m[off:off + size])) for o, s, off, size in self.index[i]]

    def __getitem__(self, i):
        if not 0 <= i < len(self):
            raise IndexError(i)
        return [self._frame(j) for j in ((i, i + self.lead) if self.lead else (i,))]

    def __getstate__(self):
        state = dict(self.__dict__)
        state["_map"] = None
        return state


@dataclass
class ChunkBatch:
    """One batch of container chunks on the wire: the archives packed on
    16-byte boundaries in one uint8 tensor, and per chunk (side, sample,
    origin, shape, offset, size)."""
    payload: object
    chunks: list
    count: int

    def pin_memory(self):
        return ChunkBatch(self.payload.pin_memory(), self.chunks, self.count)


def pack_chunks(samples):
    import torch
    data, chunks = bytearray(), []
    for i, sample in enumerate(samples):
        for side, frame in enumerate(sample):
            for origin, shape, blob in frame:
                data.extend(b"\0" * (-len(data) % 16))
                chunks.append((side, i, origin, shape, len(data), len(blob)))
                data.extend(blob)
    payload = torch.frombuffer(data, dtype=torch.uint8) if data else torch.empty(0, dtype=torch.uint8)
    return ChunkBatch(payload, chunks, len(samples))


class _Decoder:
    """Upload on a copy stream into one of two staging buffers, then decode
    the whole batch with one batched call on the caller's stream."""

    def __init__(self, dataset, device, mode):
        import torch
        self.torch = torch
        self.d = dataset
        self.device = device
        self.mode = mode
        self.copy = torch.cuda.Stream(device)
        self.staging = [None, None]
        self.slot = 0
        self.dtype = torch.float32 if dataset.width == 4 else torch.float64

    def upload(self, batch):
        torch = self.torch
        slot = self.slot
        self.slot ^= 1
        n = batch.payload.numel()
        buf = self.staging[slot]
        if buf is None or buf.numel() < n:
            buf = self.staging[slot] = torch.empty(max(n, 16), dtype=torch.uint8, device=self.device)
        # the previous user of this buffer (the batch before last) is decoded
        self.copy.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.copy):
            buf[:n].copy_(batch.payload, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.copy)
        return buf, ev

    def decode(self, batch, staged):
        torch = self.torch
        buf, ev = staged
        d = self.d
        caller = torch.cuda.current_stream(self.device)
        caller.wait_event(ev)
        sides = 2 if d.lead else 1
        outs = torch.empty((sides, batch.count, *d.shape), dtype=self.dtype, device=self.device)
        fz, fy, fx = d.shape
        covered = {}
        for side, i, o, s, off, size in batch.chunks:
            covered[(side, i)] = covered.get((side, i), 0) + math.prod(s)
        for side in range(sides):
            for i in range(batch.count):
                if covered.get((side, i), 0) != fz * fy * fx:
                    outs[side, i].fill_(d.fill)
        width = d.width
        if self.mode == "serial":
            from . import decompress_tensor
            for side, i, o, s, off, size in batch.chunks:
                arc = buf[off:off + size]
                tile = decompress_tensor(arc, s, self.dtype)
                outs[side, i, o[0]:o[0] + s[0], o[1]:o[1] + s[1], o[2]:o[2] + s[2]].copy_(tile)
        elif batch.chunks:
            items = (Archive * len(batch.chunks))()
            host = batch.payload.data_ptr()
            base = outs.data_ptr()
            end = base + outs.numel() * width
            for k, (side, i, o, s, off, size) in enumerate(batch.chunks):
                at = base + (((side * batch.count + i) * fz + o[0]) * fy * fx + o[1] * fx + o[2]) * width
                # header: the host copy of the archive in the payload tensor
                items[k] = Archive(buf.data_ptr() + off, size, host + off, s[2], s[1], s[0], at, end - at, fx, fx * fy)
            from . import autotune
            autotune.apply_batch(lib(), [s for _, _, _, s, _, _ in batch.chunks], width)
            checked(lib().waltz_b200_decompress_batch(items, len(batch.chunks), width, C.c_void_p(caller.cuda_stream)))
        return (outs[0], outs[1]) if d.lead else outs[0]


class WaltzGPUDataLoader:
    """Yield CUDA tensors of frames from a chunk container without any CPU
    decoding: (batch, z, y, x), or (input, target) pairs `lead` frames apart.
    Arguments follow the reference loader (python/pywaltz/gpu_dataloader.py:
    136-158); `key` and `library` are accepted for signature compatibility
    (the library comes from WALTZ_B200_LIBRARY or the package). decode_mode
    "batch"/"auto" decodes a batch in one call; "serial" one chunk at a time."""

    def __init__(self, path, key=None, *, device="cuda", library=None, lead=0, batch_size=1, num_workers=0,
                 pin_memory=True, shuffle=False, sampler=None, drop_last=False, persistent_workers=False,
                 decode_mode="auto"):
        import torch
        from torch.utils.data import DataLoader
        if decode_mode not in ("auto", "batch", "serial"):
            raise ValueError("decode_mode must be auto, batch or serial")
        if batch_size is None:
            raise ValueError("an integer batch_size is required")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("a CUDA device is required")
        if library is not None:
            os.environ.setdefault("WALTZ_B200_LIBRARY", os.fspath(library))
        self.mode = "serial" if decode_mode == "serial" else "batch"
        self.dataset = ChunkedFrames(path, lead)
        self._io = DataLoader(self.dataset, batch_size=batch_size, num_workers=num_workers, shuffle=shuffle,
                              sampler=sampler, drop_last=drop_last, collate_fn=pack_chunks, pin_memory=pin_memory,
                              multiprocessing_context="spawn" if num_workers else None,
                              persistent_workers=persistent_workers)

    def __len__(self):
        return len(self._io)

    def __iter__(self):
        import torch
        from torch.utils.data import get_worker_info
        if get_worker_info() is not None:
            raise RuntimeError("iterate the GPU DataLoader in the training process")
        device = self.device if self.device.index is not None else torch.device("cuda", torch.cuda.current_device())
        with torch.cuda.device(device):
            decoder = _Decoder(self.dataset, device, self.mode)
            batches = iter(self._io)
            nxt = next(batches, None)
            staged = decoder.upload(nxt) if nxt is not None else None
        while nxt is not None:
            with torch.cuda.device(device):
                cur, cur_staged = nxt, staged
                nxt = next(batches, None)
                if nxt is not None:  # the next upload overlaps this decode
                    staged = decoder.upload(nxt)
                result = decoder.decode(cur, cur_staged)
            yield result
