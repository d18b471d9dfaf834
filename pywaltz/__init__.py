"""Drop-in ``pywaltz`` surface on the B200 codec.

Code written against the reference's Python package (python/pywaltz of the
reference project) runs unchanged on this one: ``pywaltz.compress`` /
``pywaltz.decompress`` keep the reference's signatures and archives
(python/pywaltz/codec.py:65-98) but run on the current CUDA device,
``pywaltz.gpu_dataloader.WaltzGPUDataLoader`` keeps the loader's arguments,
and ``pywaltz.hdf5`` keeps filter 61197's client data. There is no CPU
fallback: without a CUDA device every codec call raises.
"""

from .codec import compress, decompress

__all__ = ["compress", "decompress"]
