"""Golden fixtures written by the reference CPU codec (see make_golden.py).

Inputs are regenerated deterministically and checked against their recorded
SHA-256 before use, so a changed generator fails loudly instead of silently
comparing different data."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

CASES = [
    {"name": "sinusoids_64_f32_rel1e-3", "kind": "sinusoids", "shape": [64, 64, 64], "seed": 0,
     "dtype": "float32", "rel": 1e-3},
    {"name": "powerlaw_40x44x52_f32_rel1e-4", "kind": "powerlaw", "shape": [40, 44, 52], "seed": 1,
     "dtype": "float32", "rel": 1e-4},
    {"name": "front_12x20x36_f64_abs1e-6", "kind": "front", "shape": [12, 20, 36], "seed": 2,
     "dtype": "float64", "abs": 1e-6},
    {"name": "pattern3_23x19x17_f64_abs1e-5", "kind": "pattern", "shape": [23, 19, 17], "pattern": 3,
     "dtype": "float64", "abs": 1e-5},
    {"name": "pattern2_9x32x48_f32_abs1e-3", "kind": "pattern", "shape": [9, 32, 48], "pattern": 2,
     "dtype": "float32", "abs": 1e-3},
    {"name": "pattern1_64_f32_abs1e-5_qoutliers", "kind": "pattern", "shape": [64, 64, 64], "pattern": 1,
     "dtype": "float32", "abs": 1e-5},
    {"name": "pattern4_5x3x2_f32_abs1e-3", "kind": "pattern", "shape": [5, 3, 2], "pattern": 4,
     "dtype": "float32", "abs": 1e-3},
    {"name": "spiky_16x40x48_f32_rel1e-5", "kind": "spiky", "shape": [16, 40, 48], "seed": 3,
     "dtype": "float32", "rel": 1e-5},
]


def make_input(case):
    from tests import patterns
    from waltz_b200 import synthetic as S
    dtype = np.dtype(case["dtype"])
    shape = tuple(case["shape"])
    kind = case["kind"]
    if kind == "sinusoids":
        field = S.sinusoids(shape, seed=case["seed"], dtype=dtype)
    elif kind == "powerlaw":
        field = S.power_law_field(shape, case["seed"], dtype=dtype)
    elif kind == "front":
        base = S.power_law_field(shape, case["seed"], slope=-5.0 / 3.0, dtype=np.float64)
        z = np.arange(shape[0], dtype=np.float64)[:, None, None]
        field = (base + 10.0 * np.tanh((z - shape[0] / 2) / 2.0)).astype(dtype)
    elif kind == "spiky":
        field = S.spiky_field(shape, case["seed"], dtype=dtype)
    else:
        field = patterns.codec_field(shape, case["pattern"], case["abs"], dtype)
    eb = case["abs"] if "abs" in case else S.rel_to_abs(field, case["rel"])
    return field, eb


def load_golden():
    meta = json.loads((HERE / "cases.json").read_text())
    blobs = np.load(HERE / "archives.npz")
    out = []
    for m in meta:
        field, eb = make_input(m)
        digest = hashlib.sha256(field.tobytes()).hexdigest()
        if digest != m["input_sha256"]:
            raise AssertionError(f"golden input generator changed for {m['name']}")
        assert eb == m["abs_error"], m["name"]
        out.append({"name": m["name"], "input": field, "abs_error": eb,
                    "archive": blobs[m["name"]].tobytes(), "decoded_sha256": m["decoded_sha256"]})
    return out
