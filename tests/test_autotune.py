"""Tuning table lookup (no GPU): classes, nearest entry, defaults."""
from __future__ import annotations

import json

from waltz_b200 import autotune as A


def test_classes():
    assert A.single_class((512, 512, 512), 4) == {"kind": "single", "dtype": "f32", "schedule": "dyadic", "log2n": 27}
    assert A.single_class((64, 1024, 1024), 4)["schedule"] == "plane"
    c = A.batch_class([(32, 32, 32)] * 512, 8)
    assert c == {"kind": "batch", "dtype": "f64", "log2count": 9, "log2mean": 15}


def test_lookup_nearest_and_defaults(tmp_path):
    table = {"entries": [
        {"class": {"kind": "single", "dtype": "f32", "schedule": "dyadic", "log2n": 18},
         "choice": {"stage_kernels": 1, "zmarch": 32}},
        {"class": {"kind": "single", "dtype": "f32", "schedule": "dyadic", "log2n": 27},
         "choice": {"stage_kernels": 1, "zmarch": 0}},
        {"class": {"kind": "batch", "dtype": "f32", "log2count": 9, "log2mean": 18},
         "choice": {"mode": 0, "width": 4, "stage_kernels": 0}},
    ]}
    path = tmp_path / "t.json"
    path.write_text(json.dumps(table))
    assert A.lookup(A.single_class((64, 64, 64), 4), path)["zmarch"] == 32
    assert A.lookup(A.single_class((400, 400, 400), 4), path)["zmarch"] == 0
    # no plane-schedule or f64 entry: defaults
    assert A.lookup(A.single_class((32, 128, 128), 4), path) == A.DEFAULT_SINGLE
    assert A.lookup(A.single_class((64, 64, 64), 8), path) == A.DEFAULT_SINGLE
    assert A.lookup(A.batch_class([(64, 64, 64)] * 300, 4), path) == {"mode": 0, "width": 4, "stage_kernels": 0}
    assert A.lookup(A.batch_class([(64, 64, 64)] * 300, 8), path) == A.DEFAULT_BATCH


def test_committed_table_is_well_formed():
    t = A.load()
    for e in t.get("entries", []):
        assert e["class"]["kind"] in ("single", "batch")
        assert e["measured"] and all(r["compress_ms"] > 0 and r["decompress_ms"] > 0 for r in e["measured"])
        best = min(e["measured"], key=lambda r: r["compress_ms"] + r["decompress_ms"])["knobs"]
        assert all(e["choice"][k] == v for k, v in best.items())


def test_matrix_choice_follows_the_rule():
    """Entries that timed the precision-form splits choose the fastest
    candidate (double fields: the exact slices only) that beats the plain
    knobs by the margin with an archive at most 2 % larger than the plain
    one, or none."""
    t = A.load()
    for e in t.get("entries", []):
        if "matrix_forms" not in e:
            continue
        itemsize = 4 if e["class"]["dtype"] == "f32" else 8
        best = min(e["measured"], key=lambda r: r["compress_ms"] + r["decompress_ms"])
        limit = A.MATRIX_MARGIN * (best["compress_ms"] + best["decompress_ms"])
        ok = sorted((m["compress_ms"] + m["decompress_ms"], f) for f, m in e["matrix_forms"].items()
                    if f in A.matrix_candidates(itemsize) and m["compress_ms"] + m["decompress_ms"] < limit
                    and m["archive_bytes"] * A.MATRIX_RATIO <= e["plain_archive_bytes"])
        assert e["choice"]["matrix"] == (ok[0][1] if ok else False)
        assert A.choose_matrix(e, itemsize) == e["choice"]["matrix"]
        if itemsize == 8:
            assert e["choice"]["matrix"] in (False, "matrix-exact")


def test_matrix_choice_lookup(tmp_path):
    table = {"entries": [
        {"class": {"kind": "single", "dtype": "f32", "schedule": "plane", "log2n": 26},
         "choice": {"stage_kernels": 1, "matrix": "matrix-bf16"}},
        {"class": {"kind": "single", "dtype": "f64", "schedule": "plane", "log2n": 23},
         "choice": {"stage_kernels": 1, "matrix": False}},
    ]}
    path = tmp_path / "t.json"
    path.write_text(json.dumps(table))
    assert A.matrix_choice((64, 1024, 1024), 4, path) == "matrix-bf16"
    assert A.matrix_choice((96, 256, 384), 8, path) is None
    assert A.matrix_choice((512, 512, 512), 4, path) is None  # dyadic: no entry of that schedule
