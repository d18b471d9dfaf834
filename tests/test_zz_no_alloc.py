"""The allocation-free WZP encoder (waltz_b200_wzp_encode_noalloc).

It serves callers that cannot allocate device memory when they call (a host
framework whose allocator owns the device budget, a plugin callback, a loop
that cannot take cudaMalloc's device synchronisation). Its working state is a
static device array shared by every call, so these tests check that two
calls in a row, each reusing the previous call's leftovers, write exactly
the stream of the allocating encoder. The file sorts last so that a run that
stops at its first failure has run every other test before this one.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tests import patterns as P

pytestmark = pytest.mark.gpu

NOALLOC_MAX = 16384 * 8192


def _encode(fn_name, dm, ds, n, cap):
    import torch
    from waltz_b200 import _lib
    lib = _lib.lib()
    out = torch.full((cap,), 0xA5, dtype=torch.uint8, device="cuda")
    written = C.c_size_t()
    rc = getattr(lib, fn_name)(C.c_void_p(dm.data_ptr()), C.c_void_p(ds.data_ptr()), n, C.c_void_p(out.data_ptr()),
                               cap, C.byref(written), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.last_error()
    return out[:written.value].cpu().numpy().tobytes()


def _device(mag, sign):
    import torch
    return (torch.from_numpy(mag.astype(np.uint16).view(np.int16)).cuda(),
            torch.from_numpy(sign.astype(np.uint32).view(np.int32)).cuda())


def test_noalloc_matches_allocating_encoder_twice_in_a_row():
    """Every WZP test case: two allocation-free calls in a row, each equal to
    the allocating encoder's stream."""
    for n, pattern, mag, sign in P.wzp_cases():
        if n == 0:
            continue
        dm, ds = _device(mag, sign)
        cap = 4 * 1024 + 3 * n
        expect = _encode("waltz_b200_wzp_encode", dm, ds, n, cap)
        first = _encode("waltz_b200_wzp_encode_noalloc", dm, ds, n, cap)
        second = _encode("waltz_b200_wzp_encode_noalloc", dm, ds, n, cap)
        assert first == expect, (n, pattern)
        assert second == expect, (n, pattern)


def test_noalloc_at_the_size_limit_then_small():
    """A call at the maximum size (16384 chunks) and a small call right after
    it, whose lookback states must not see the large call's leftovers."""
    rng = np.random.default_rng(11)
    for n in (NOALLOC_MAX, 3 * 8192 + 5):
        mag = np.where(rng.random(n) < 0.3, rng.integers(0, 65536, n), 0).astype(np.uint16)
        sign = rng.integers(0, 2 ** 32, (n + 31) // 32, dtype=np.uint64).astype(np.uint32)
        dm, ds = _device(mag, sign)
        cap = 4 * 1024 + 3 * n
        expect = _encode("waltz_b200_wzp_encode", dm, ds, n, cap)
        for _ in range(2):
            assert _encode("waltz_b200_wzp_encode_noalloc", dm, ds, n, cap) == expect, n


def test_noalloc_rejects_sizes_beyond_its_limit():
    """n above the limit is refused on the host with a clear error, before
    any device work."""
    import torch
    from waltz_b200 import _lib
    lib = _lib.lib()
    dm = torch.zeros(16, dtype=torch.int16, device="cuda")
    ds = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros(64, dtype=torch.uint8, device="cuda")
    written = C.c_size_t(123)
    rc = lib.waltz_b200_wzp_encode_noalloc(C.c_void_p(dm.data_ptr()), C.c_void_p(ds.data_ptr()), NOALLOC_MAX + 1,
                                           C.c_void_p(out.data_ptr()), 64, C.byref(written),
                                           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc != 0 and written.value == 0
    assert "allocation-free limit" in _lib.last_error()
