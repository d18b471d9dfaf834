"""The reference loader's wire format (python/pywaltz/_raw_chunks.py:97-125 of
the reference project): archive blobs on 16-byte boundaries followed by
(u64 offset, u64 size) spans, decoded by ``waltz_gpu_decode_batch``."""

from waltz_b200.loader import WireBatch, decode_batch, pack

__all__ = ["WireBatch", "pack", "decode_batch"]
