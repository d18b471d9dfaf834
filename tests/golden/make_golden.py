"""Regenerate the golden fixtures from the reference CPU codec itself
(oracle/_ref/libwaltz_ref.so, compiled from the reference sources by
`make -C oracle ref`). Run from the repository root:

    python tests/golden/make_golden.py

Each case records how its input is generated (a seeded synthetic field or a
reference test pattern), the input's SHA-256, the bound, the archive bytes
written by the reference scalar codec and the SHA-256 of its decode.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from tests.golden import CASES, make_input  # noqa: E402

HERE = Path(__file__).resolve().parent


def main():
    ref = O.RefCodec(O.SCALAR)
    meta = []
    blobs = {}
    for case in CASES:
        field, eb = make_input(case)
        archive = ref.compress(field, eb)
        decoded = ref.decompress(archive, field.shape, field.dtype)
        meta.append({**case, "abs_error": eb, "input_sha256": hashlib.sha256(field.tobytes()).hexdigest(),
                     "archive_bytes": len(archive),
                     "decoded_sha256": hashlib.sha256(decoded.tobytes()).hexdigest()})
        blobs[case["name"]] = np.frombuffer(archive, np.uint8)
        print(f"{case['name']}: {field.shape} {field.dtype} eb={eb:.6g} archive={len(archive)}")
    np.savez_compressed(HERE / "archives.npz", **blobs)
    (HERE / "cases.json").write_text(json.dumps(meta, indent=1) + "\n")


if __name__ == "__main__":
    main()
