"""Deterministic test inputs restating the reference test generators
(cpu/tests/test_codec.cpp:68-91 fill patterns, cpu/tests/test_wzp.cpp:197-223
WZP patterns): xorshift32 streams and closed-form fields."""
from __future__ import annotations

import math

import numpy as np


def xorshift_stream(state: int, count: int) -> tuple[np.ndarray, int]:
    out = np.empty(count, np.uint32)
    s = state
    for i in range(count):
        s ^= (s << 13) & 0xffffffff
        s ^= s >> 17
        s ^= (s << 5) & 0xffffffff
        out[i] = s
    return out, s


def codec_field(shape_zyx, pattern: int, abs_error: float, dtype) -> np.ndarray:
    """Field of the reference codec acceptance test for pattern 0..6."""
    nz, ny, nx = shape_zyx
    n = nx * ny * nz
    rng, _ = xorshift_stream(0x1879B52D, n)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i = np.arange(n).reshape(shape_zyx)
    if pattern == 0:
        v = np.zeros(shape_zyx)
    elif pattern == 1:
        v = np.full(shape_zyx, 1.25)
    elif pattern == 2:
        v = np.sin(0.17 * x) + np.cos(0.21 * y) - 0.03 * z
        v = v + np.where((x + 3 * y + 7 * z) % 19 == 0, 0.125, 0.0)
    elif pattern == 3:
        v = ((rng & 0x00FFFFFF).astype(np.float64) / 0x01000000 - 0.5).reshape(shape_zyx) * 2
    elif pattern == 4:
        v = np.where((x + y + z) & 1, -4.0, 4.0)
        v.reshape(-1)[0] = 32
        v.reshape(-1)[-1] = -32
    elif pattern == 5:
        v = np.where(i % 7 == 0, -0.0, ((i % 9).astype(np.float64) - 4) * abs_error * 0.499)
    else:
        v = 1048576.0 + ((i % 33).astype(np.float64) - 16) * 0.125
    return v.astype(dtype)


WZP_SIZES = [0, 1, 2, 7, 8, 15, 16, 17, 31, 32, 33, 63, 127, 255, 256, 511, 8191, 8192, 8193, 16384,
             15 * 8192 + 7, 16 * 8192, 16 * 8192 + 1, 32 * 8192 + 37]


def wzp_cases():
    """(n, pattern, mag u16[n], sign u32[ceil(n/32)]) of the reference WZP test."""
    state = 0x728CA19B
    for n in WZP_SIZES:
        words = (n + 31) // 32
        for pattern in range(8):
            signs, state = xorshift_stream(state, words)
            r, state = xorshift_stream(state, n)
            i = np.arange(n, dtype=np.uint64)
            if pattern == 0:
                m = np.zeros(n, np.uint32)
            elif pattern == 1:
                m = np.ones(n, np.uint32)
            elif pattern == 2:
                m = r & 0xFFFF
            elif pattern == 3:
                m = np.where(r % 97 == 0, r >> 16, 0)
            elif pattern == 4:
                m = r & 7
            elif pattern == 5:
                m = np.where((i // 8192) % 3 == 0, 0, r & 0xFFFF)
            elif pattern == 6:
                m = np.where(i % 16 == 0, 0x8000, 0)
            else:
                m = np.where((i // (16 * 8192)) % 2 == 0, 0, 0xFFFF)
            yield n, pattern, m.astype(np.uint16), signs.astype(np.uint32)


CODEC_SHAPES = [(1, 1, 1), (2, 3, 5), (8, 8, 8), (16, 16, 16), (17, 19, 23), (48, 32, 9), (9, 11, 65),
                (1, 17, 33), (33, 31, 17), (64, 64, 64)]  # (nx, ny, nz) as in the reference test


def zyx(nxyz):
    nx, ny, nz = nxyz
    return (nz, ny, nx)
