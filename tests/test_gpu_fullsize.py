"""GPU: the full-size configurations pinned to the reference CPU codec.

The plain form's archive of each full-size field is compared byte for byte
with the reference CPU codec's (oracle/_ref, its AVX2 backend, whose bytes
equal its scalar backend's: cpu/tests/test_codec.cpp:161-181 of the
reference), and the GPU decode bit for bit with the CPU decode of the same
archive; every sample stays within the bound. This is the reference's own
GPU/CPU interop check (cpu/tests/interop_gpu.cu:159-268) at the sizes the
benchmark runs:

* f32 512^3 k^-11/3 Gaussian random field (seed 1), dyadic 5 levels,
  REL 1e-3 and REL 1e-4;
* f32 1024x1024x64 k^-11/3 field (seed 3) with 1 % spikes of +-50, plane
  schedule (5 XY / 3 Z levels), REL 1e-3 and REL 1e-5.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="reference CPU codec not built (oracle/Makefile ref)")]

_FIELDS = {}


def _field(name):
    import torch
    from waltz_b200 import synthetic as S
    if name not in _FIELDS:
        _FIELDS.clear()
        torch.cuda.empty_cache()
        if name == "grf512":
            _FIELDS[name] = S.power_law_field_device((512, 512, 512), 1).contiguous()
        else:
            _FIELDS[name] = S.spiky_field_device((64, 1024, 1024), 3)
    return _FIELDS[name]


@pytest.mark.parametrize("name,rel", [("grf512", 1e-3), ("grf512", 1e-4), ("spiky1024x1024x64", 1e-3),
                                      ("spiky1024x1024x64", 1e-5)])
def test_full_size_archive_identical_to_cpu_codec(name, rel):
    import torch
    import waltz_b200
    d = _field(name)
    lo, hi = waltz_b200.extrema(d)
    eb = rel * (hi - lo)
    host = d.cpu().numpy()
    assert (float(host.min()), float(host.max())) == (lo, hi)
    archive_d = waltz_b200.compress_tensor(d, eb, tuned=False)
    archive = archive_d.cpu().numpy().tobytes()
    ref = O.RefCodec(O.AVX2)
    expect = ref.compress(host, eb)
    assert len(archive) == len(expect)
    assert archive == expect
    out = waltz_b200.decompress_tensor(archive_d, tuple(d.shape), torch.float32, tuned=False)
    cpu_out = ref.decompress(expect, host.shape, np.float32)
    got = out.cpu().numpy()
    assert got.tobytes() == cpu_out.tobytes()
    err = float(np.abs(got.astype(np.float64) - host.astype(np.float64)).max())
    assert err <= eb
