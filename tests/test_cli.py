"""The command-line codec (waltz_b200.cli), whose options follow the
reference's examples/waltz.cu: argument handling and statistics on the CPU,
the file round trip against the oracle on the GPU."""
from __future__ import annotations

import math

import numpy as np
import pytest

from waltz_b200 import cli


def test_parse_compress_and_temporary_archive():
    a = cli.parse(["-f", "-i", "in.f32", "-z", "c.waltz", "-3", "8", "9", "10", "-M", "REL", "1e-3"])
    assert (a.dtype, a.input, a.compressed, a.output, a.dims, a.bound) == ("f32", "in.f32", "c.waltz", None,
                                                                           [8, 9, 10], 1e-3)
    # -i with -o and no -z: the archive goes to <input>.waltz.tmp (examples/waltz.cu:254-259)
    a = cli.parse(["-d", "-i", "in.f64", "-o", "out.f64", "-3", "4", "4", "4", "-M", "ABS", "0.5"])
    assert (a.dtype, a.compressed, a.output, a.bound) == ("f64", "in.f64.waltz.tmp", "out.f64", 0.5)


def test_parse_decompress_forms():
    a = cli.parse(["-z", "c.waltz", "-o", "o.f32", "-3", "2", "3", "4"])
    assert (a.mode, a.compressed, a.output) == (None, "c.waltz", "o.f32")
    a = cli.parse(["-i", "c.waltz", "-o", "o.f32", "-3", "2", "3", "4"])
    assert (a.mode, a.input, a.output) == (None, "c.waltz", "o.f32")


@pytest.mark.parametrize("argv", [
    ["-i", "x", "-z", "y", "-M", "REL", "1e-3"],                      # no dimensions
    ["-i", "x", "-z", "y", "-3", "0", "4", "4", "-M", "REL", "1e-3"],  # empty dimension
    ["-i", "x", "-z", "y", "-3", "4", "4", "4", "-M", "PSNR", "60"],   # unsupported mode
    ["-i", "x", "-z", "y", "-3", "4", "4", "4", "-M", "ABS", "0"],     # non-positive bound
    ["-i", "x", "-z", "y", "-3", "4", "4", "4", "-M", "ABS", "nan"],
    ["-i", "x", "-3", "4", "4", "4", "-M", "ABS", "1"],                # nowhere to write
    ["-z", "y", "-3", "4", "4", "4"],                                  # decode without -o
    ["-f", "-d", "-z", "y", "-o", "o", "-3", "4", "4", "4"],           # two sample types
])
def test_parse_rejects(argv, capsys):
    with pytest.raises(SystemExit) as e:
        cli.parse(argv)
    assert e.value.code == 2


def test_stats_match_definition():
    orig = np.array([0.0, 1.0, 2.0, 4.0], dtype=np.float32)
    rec = np.array([0.0, 1.5, 2.0, 3.75], dtype=np.float32)
    st = cli.stats(orig, rec)
    mse = (0.25 + 0.0625) / 4
    assert st["max_abs_error"] == 0.5 and st["index"] == 1
    assert st["max_rel_error"] == 0.5 / 4
    assert math.isclose(st["psnr_db"], 20 * math.log10(4) - 10 * math.log10(mse))
    assert math.isclose(st["nrmse"], math.sqrt(mse) / 4)
    with pytest.raises(ValueError):
        cli.stats(np.zeros(0, np.float32), np.zeros(0, np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,flag", [(np.float32, "-f"), (np.float64, "-d")])
@pytest.mark.parametrize("mode,bound", [("REL", 1e-3), ("ABS", 0.05)])
def test_cli_round_trip_matches_oracle(tmp_path, capsys, dtype, flag, mode, bound):
    from oracle import oracle as O
    nx, ny, nz = 40, 33, 21
    rng = np.random.default_rng(5)
    data = np.cumsum(rng.standard_normal((nz, ny, nx)), axis=2).astype(dtype)
    src, arc, out = tmp_path / "f.raw", tmp_path / "f.waltz", tmp_path / "f.out"
    data.tofile(src)
    assert cli.main([flag, "-i", str(src), "-z", str(arc), "-3", str(nx), str(ny), str(nz), "-M", mode,
                     str(bound), "-o", str(out)]) == 0
    eb = bound * (float(data.max()) - float(data.min())) if mode == "REL" else bound
    expect = O.compress(data, eb)
    assert arc.read_bytes() == expect
    rec = np.fromfile(out, dtype=dtype)
    assert rec.tobytes() == O.decompress(expect, data.shape, dtype).tobytes()
    assert np.abs(rec.astype(np.float64) - data.ravel().astype(np.float64)).max() <= eb
    printed = capsys.readouterr().out
    assert "Compression Ratio" in printed and "PSNR" in printed
    # decode alone, from the archive file
    out2 = tmp_path / "g.out"
    assert cli.main([flag, "-z", str(arc), "-o", str(out2), "-3", str(nx), str(ny), str(nz)]) == 0
    assert out2.read_bytes() == out.read_bytes()
