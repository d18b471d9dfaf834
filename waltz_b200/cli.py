"""Command-line codec on the GPU, with the options of the reference's
`waltz` example (examples/waltz.cu:11-35):

  Compress:   python -m waltz_b200 [-f|-d] -i input -z compressed -3 nx ny nz -M REL|ABS bound [-o output]
  Decompress: python -m waltz_b200 [-f|-d] -z compressed -o output -3 nx ny nz
              (-i compressed -o output also works without -M)

-f / -d select float32 (default) / float64. Raw files hold nx*ny*nz samples,
x fastest. REL resolves to REL * (max - min) on the GPU before compressing
(examples/waltz.cu:50-55). With -o during compression the reconstruction is
written and compared with the input (max error, PSNR, ratio). --form matrix,
matrix-bf16 or matrix-exact selects the precision form (its tensor-core
split); WALTZ_WARMUP=1 runs each call once untimed and
WALTZ_REPORT_CE2E=1 prints the device time of the call, as in the reference.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np


def parse(argv):
    ap = argparse.ArgumentParser(prog="python -m waltz_b200", add_help=True,
                                 description="Waltz error-bounded compressor on the GPU (B200)")
    t = ap.add_mutually_exclusive_group()
    t.add_argument("-f", dest="dtype", action="store_const", const="f32", help="float32 samples (default)")
    t.add_argument("-d", dest="dtype", action="store_const", const="f64", help="float64 samples")
    ap.add_argument("-i", dest="input", help="raw input (compress) or compressed input (decode without -M)")
    ap.add_argument("-z", dest="compressed", help="compressed output (compress) or input (decode)")
    ap.add_argument("-o", dest="output", help="reconstruction; with compression also verified against the input")
    ap.add_argument("-3", dest="dims", nargs=3, type=int, metavar=("NX", "NY", "NZ"), required=True)
    ap.add_argument("-M", dest="mode", nargs=2, metavar=("REL|ABS", "BOUND"))
    ap.add_argument("--form", choices=["plain", "matrix", "matrix-bf16", "matrix-exact", "auto"], default="plain")
    a = ap.parse_args(argv)
    a.dtype = a.dtype or "f32"
    if any(v <= 0 for v in a.dims):
        ap.error("dimensions must be positive")
    if a.mode:
        if a.mode[0].upper() not in ("REL", "ABS"):
            ap.error("-M takes REL or ABS")
        try:
            a.bound = float(a.mode[1])
        except ValueError:
            ap.error("invalid error bound")
        if not (math.isfinite(a.bound) and a.bound > 0):
            ap.error("the error bound must be positive and finite")
        if not a.input:
            ap.error("compression needs -i input")
        if not a.compressed:
            if not a.output:
                ap.error("compression needs -z compressed (or -o output)")
            a.compressed = a.input + ".waltz.tmp"  # examples/waltz.cu:254-259
    else:
        src = a.compressed or a.input
        if not src or not a.output:
            ap.error("decompression needs -z compressed (or -i compressed) and -o output")
    return a


def _timed(torch, fn):
    warm = os.environ.get("WALTZ_WARMUP", "0") not in ("", "0")
    if warm:
        fn()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    out = fn()
    end.record()
    torch.cuda.synchronize()
    return out, start.elapsed_time(end)


def _report(name, nbytes, ms):
    if os.environ.get("WALTZ_REPORT_CE2E", "0") not in ("", "0"):
        print(f"{name}: {ms:.3f} ms, {nbytes / (ms / 1e3) / 1e9:.2f} GB/s")


def stats(orig, rec):
    """Error statistics of a reconstruction, as include/utils/Statistics.hpp:206
    reports them: the difference taken in the sample type, then in double."""
    if orig.size == 0:
        raise ValueError("statistics need at least one sample")
    err = np.abs((rec.ravel() - orig.ravel()).astype(np.float64))
    idx = int(np.argmax(err))
    rng = float(orig.max()) - float(orig.min())
    mse = float(np.mean(err * err))
    with np.errstate(divide="ignore", invalid="ignore"):
        psnr = float(20 * np.log10(np.float64(rng)) - 10 * np.log10(np.float64(mse)))
        nrmse = float(np.sqrt(mse) / np.float64(rng))
        max_re = float(err[idx] / np.float64(rng))
    return {"max_abs_error": float(err[idx]), "index": idx, "max_rel_error": max_re, "psnr_db": psnr,
            "nrmse": nrmse}


def print_stats(st):
    print(f"  Max_E  = {st['max_abs_error']:.15f}, idx = {st['index']}")
    print(f"  Max_RE = {st['max_rel_error']:G}")
    print(f"  PSNR = {st['psnr_db']:.7f}, NRMSE = {st['nrmse']:.10G}")


def main(argv=None):
    a = parse(sys.argv[1:] if argv is None else argv)
    import torch
    import waltz_b200
    np_dtype = np.float32 if a.dtype == "f32" else np.float64
    nx, ny, nz = a.dims
    shape = (nz, ny, nx)
    n = nx * ny * nz
    if a.mode:
        data = np.fromfile(a.input, dtype=np_dtype)
        if data.size != n:
            raise SystemExit(f"{a.input}: {data.size} samples, expected {n}")
        field = torch.from_numpy(data.reshape(shape)).cuda()
        eb = a.bound
        if a.mode[0].upper() == "REL":
            eb = waltz_b200.rel_to_abs_bound(field, a.bound)
        archive, ms = _timed(torch, lambda: waltz_b200.compress_tensor(field, eb, form=a.form))
        _report("compress", n * data.itemsize, ms)
        blob = archive.cpu().numpy().tobytes()
        with open(a.compressed, "wb") as fh:
            fh.write(blob)
        print(f"  {'Compression Ratio':<17} = {n * data.itemsize / len(blob):.5f}")
        del field, archive
        if a.output:
            decode(torch, waltz_b200, a.compressed, a.output, shape, np_dtype)
            rec = np.fromfile(a.output, dtype=np_dtype)
            print_stats(stats(data, rec))
        return 0
    decode(torch, waltz_b200, a.compressed or a.input, a.output, shape, np_dtype)
    return 0


def decode(torch, waltz_b200, src, dst, shape, np_dtype):
    with open(src, "rb") as fh:
        blob = fh.read()
    if len(blob) < 32:
        raise SystemExit("Cannot read compressed file or header is incomplete")
    archive = torch.frombuffer(bytearray(blob), dtype=torch.uint8).cuda()
    dtype = torch.float32 if np_dtype == np.float32 else torch.float64
    out, ms = _timed(torch, lambda: waltz_b200.decompress_tensor(archive, shape, dtype))
    nbytes = out.numel() * out.element_size()
    _report("decompress", nbytes, ms)
    out.cpu().numpy().tofile(dst)
    print(f"  {'Compression Ratio':<17} = {nbytes / len(blob):.5f}")


if __name__ == "__main__":
    sys.exit(main())
