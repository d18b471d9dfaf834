"""``WaltzGPUDataLoader`` under the reference's module path
(python/pywaltz/gpu_dataloader.py:136-181 of the reference project), with its
arguments. Frames come from the chunk container of ``waltz_b200.loader``
(``write_frames``); every batch decodes on the GPU in one call."""

from waltz_b200.loader import ChunkedFrames, WaltzGPUDataLoader, write_frames

__all__ = ["WaltzGPUDataLoader", "ChunkedFrames", "write_frames"]
