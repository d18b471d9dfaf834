"""Autotuner of the codec's performance knobs, and the committed table it
writes (``tuning.json`` beside this file).

Knobs (none changes a byte of the output, so a choice is a pure timing
question and the table can be applied blindly):
 * single fields: the plane schedule's whole-stage kernels on or off
   (WALTZ_B200_OPT_STAGE_KERNELS), the forward z-march depth, the planes
   per CTA tile of the dyadic forward levels (WALTZ_B200_OPT_ZMARCH_PLANES),
   and the level sizes below which dyadic and XY levels stage tiles with
   reflecting loads instead of tensor-map copies (WALTZ_B200_OPT_SMALL_LEVEL /
   _FWD);
 * batches: the execution form of the batch graph (stage-batched groups,
   the same as persistent work queues, or per-field chains, and their width,
   waltz_b200_batch_config), the stage kernels knob and, for stage-batched
   groups, the forward z-march depth (short ranges give small chunks more
   CTAs for the price of re-read z halos), tensor-map staging on every
   level (the small-level thresholds at 0) and the plane XY levels as the
   warp march, forward and inverse levels separately
   (WALTZ_B200_OPT_XY_MARCH bits 0 and 1; single plane fields try it too),
   and the size up to which dyadic inverse levels run as a Z march and an
   XY march instead of the tile inverse (WALTZ_B200_OPT_SMALL_MARCH), and
   dyadic forward levels as an XY march and a Z march instead of the
   z-march (WALTZ_B200_OPT_SMALL_MARCH_FWD); single dyadic fields try both;
 * the transform form (lifting or one split of the tensor-core matrix form)
   of fields the matrix form serves: every split is timed and the fastest
   one that beats lifting by 3 % with a compression ratio at most 2 % lower
   is recorded per class; it is used only when a caller asks for
   form="auto", since the matrix form sets its own header flag.
The WZP group size (16 chunks of 8192 samples) is part of the archive
format the reference decoders read, so it is not a knob.

Classes: single fields by (dtype, schedule, round(log2 n)); batches by
(dtype, round(log2 count), round(log2 mean chunk size)). A lookup takes the
nearest measured class of the same dtype and kind.

Run on a GPU:  python -m waltz_b200.autotune [--quick]
"""
from __future__ import annotations

import json
import math
import statistics
import time
from pathlib import Path

TABLE = Path(__file__).with_name("tuning.json")

OPT_STAGE_KERNELS, OPT_ZMARCH_PLANES, OPT_SMALL_LEVEL, OPT_SMALL_FWD = 1, 2, 3, 4
OPT_XY_MARCH = 6
OPT_SMALL_MARCH, OPT_SMALL_MARCH_FWD = 7, 8
BATCH_STAGES, BATCH_FIELDS, BATCH_QUEUE = 0, 1, 2
DEFAULT_SINGLE = {"stage_kernels": 1, "zmarch": 0, "small_inv": 1 << 15, "small_fwd": 1 << 20, "xy_march": 0,
                  "small_march": 0, "small_march_fwd": 0}
SMALL_MARCH_CHOICES = (0, 1 << 21, 1 << 24, 1 << 27)  # dyadic inverse levels as Z + XY marches up to this size
SMALL_MARCH_FWD_CHOICES = (0, 1 << 21, 1 << 24)       # the same for dyadic forward levels
MATRIX_MARGIN = 0.97  # the matrix form changes the header flag: take it only for a clear gain
MATRIX_RATIO = 0.98   # ... and only when its archive stays within 2 % of the plain one's size
MATRIX_SPLITS = ("matrix-tf32", "matrix-bf16", "matrix-exact")


def matrix_candidates(itemsize):
    """Splits form="auto" may take: any for float fields; for double fields
    only the exact slices, since the float-accurate splits' coefficient error
    (about 1e-6 of a column's range) turns into extra repair records at the
    tight bounds double fields are compressed with (-8 % ratio at ABS 1e-4 on
    the f64 plane-schedule configuration) although a REL 1e-3 timing run does
    not see it."""
    return MATRIX_SPLITS if itemsize == 4 else ("matrix-exact",)


def choose_matrix(entry, itemsize):
    """The split an entry with timed splits takes: the fastest candidate at
    least 3 % faster than the chosen plain knobs whose archive is at most 2 %
    larger than the plain one; False when none is."""
    best = min(entry["measured"], key=lambda r: r["compress_ms"] + r["decompress_ms"])
    limit = MATRIX_MARGIN * (best["compress_ms"] + best["decompress_ms"])
    ok = sorted((m["compress_ms"] + m["decompress_ms"], form) for form, m in entry["matrix_forms"].items()
                if form in matrix_candidates(itemsize) and m["compress_ms"] + m["decompress_ms"] < limit
                and m["archive_bytes"] * MATRIX_RATIO <= entry["plain_archive_bytes"])
    return ok[0][1] if ok else False
DEFAULT_BATCH = {"mode": BATCH_FIELDS, "width": 32, "stage_kernels": 1}

SINGLE_CANDIDATES = [{"stage_kernels": s, "zmarch": z, "small_inv": i, "small_fwd": f}
                     for s in (1, 0) for z in (0, 32) for i in (1 << 15, 1 << 18, 1 << 21)
                     for f in (1 << 20, 1 << 21, 1 << 24, 1 << 26)]
BATCH_CANDIDATES = ([{"mode": BATCH_STAGES, "width": w, "stage_kernels": s, "zmarch": z, "small_inv": si, "small_fwd": sf,
                      "xy_march": xy}
                     for w in (1, 4, 16) for s in (1, 0) for z in (0, 16, 32)
                     for si, sf in ((1 << 15, 1 << 20), (0, 0)) for xy in (0, 1, 2, 3)] +
                    [{"mode": BATCH_STAGES, "width": w, "stage_kernels": s, "zmarch": z, "small_inv": 0, "small_fwd": 0,
                      "xy_march": xy, "small_march": 1 << 24, "small_march_fwd": mf}
                     for w in (4, 16) for s in (1, 0) for z in (0, 32) for xy in (0, 3) for mf in (0, 1 << 24)] +
                    [{"mode": BATCH_QUEUE, "width": w, "stage_kernels": s} for w in (1, 4, 16) for s in (1, 0)] +
                    [{"mode": BATCH_FIELDS, "width": w, "stage_kernels": s} for w in (16, 32, 64) for s in (1, 0)])


def _levels(n):
    l = 0
    while n > 8 and l < 5:
        n -= n // 2
        l += 1
    return l


def single_class(shape, itemsize):
    nz, ny, nx = shape
    sched = "dyadic" if _levels(min(nx, ny)) == _levels(nz) else "plane"
    return {"kind": "single", "dtype": "f32" if itemsize == 4 else "f64", "schedule": sched,
            "log2n": round(math.log2(max(1, nx * ny * nz)))}


def batch_class(shapes, itemsize):
    mean = sum(math.prod(s) for s in shapes) / max(1, len(shapes))
    return {"kind": "batch", "dtype": "f32" if itemsize == 4 else "f64",
            "log2count": round(math.log2(max(1, len(shapes)))), "log2mean": round(math.log2(max(1.0, mean)))}


_cache = {}


def load(path=TABLE):
    key = str(path)
    if key not in _cache:
        try:
            _cache[key] = json.loads(Path(path).read_text())
        except (OSError, ValueError):
            _cache[key] = {"entries": []}
    return _cache[key]


def lookup(cls, path=TABLE):
    """Knobs of the nearest measured class (same kind, dtype and schedule),
    or the built-in defaults."""
    best, dist = None, None
    for e in load(path).get("entries", []):
        c = e["class"]
        if c["kind"] != cls["kind"] or c["dtype"] != cls["dtype"] or c.get("schedule") != cls.get("schedule"):
            continue
        d = sum(abs(c[k] - cls[k]) for k in ("log2n", "log2count", "log2mean") if k in cls)
        if dist is None or d < dist:
            best, dist = e, d
    if best is None:
        return dict(DEFAULT_SINGLE if cls["kind"] == "single" else DEFAULT_BATCH)
    return dict(best["choice"])


def set_single(lib, k):
    """Applies single-field knobs (missing ones take their defaults)."""
    k = {**DEFAULT_SINGLE, **k}
    lib.waltz_b200_set_option(OPT_STAGE_KERNELS, int(k["stage_kernels"]))
    lib.waltz_b200_set_option(OPT_ZMARCH_PLANES, int(k["zmarch"]))
    lib.waltz_b200_set_option(OPT_SMALL_LEVEL, int(k["small_inv"]))
    lib.waltz_b200_set_option(OPT_SMALL_FWD, int(k["small_fwd"]))
    lib.waltz_b200_set_option(OPT_XY_MARCH, int(k["xy_march"]))
    lib.waltz_b200_set_option(OPT_SMALL_MARCH, int(k["small_march"]))
    lib.waltz_b200_set_option(OPT_SMALL_MARCH_FWD, int(k["small_march_fwd"]))
    return k


def apply_single(lib, shape, itemsize):
    return set_single(lib, lookup(single_class(shape, itemsize)))


def apply_batch(lib, shapes, itemsize):
    k = lookup(batch_class(shapes, itemsize))
    lib.waltz_b200_batch_config(int(k["mode"]), int(k["width"]))
    set_single(lib, batch_single_knobs(k))
    return k


def batch_single_knobs(k):
    """The single-field knobs a batch entry sets (missing ones: defaults)."""
    return {"stage_kernels": int(k.get("stage_kernels", 1)), "zmarch": int(k.get("zmarch", 0)),
            "small_inv": int(k.get("small_inv", DEFAULT_SINGLE["small_inv"])),
            "small_fwd": int(k.get("small_fwd", DEFAULT_SINGLE["small_fwd"])),
            "xy_march": int(k.get("xy_march", 0)), "small_march": int(k.get("small_march", 0)),
            "small_march_fwd": int(k.get("small_march_fwd", 0))}


def matrix_choice(shape, itemsize, path=TABLE):
    """The precision-form split the measured class takes under form="auto"
    (a form name), or None for the plain form."""
    m = lookup(single_class(shape, itemsize), path).get("matrix")
    return m if isinstance(m, str) and m in MATRIX_SPLITS else None


# ------------------------------------------------------------------ tuning
def _time(torch, fn, reps):
    fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.median(ms)


def _tune_single(torch, lib, shape, dtype, reps, rel=1e-3):
    import waltz_b200
    from .synthetic import power_law_field_device
    f = power_law_field_device(shape, 11, dtype=dtype).contiguous()
    lo, hi = waltz_b200.extrema(f)
    eb = rel * (hi - lo)
    itemsize = f.element_size()
    results = []
    # plane fields also try their XY levels as the warp march
    cands = SINGLE_CANDIDATES
    if single_class(shape, itemsize)["schedule"] == "plane":
        cands = cands + [{**c, "xy_march": xy} for xy in (1, 2, 3) for c in SINGLE_CANDIDATES]
    else:
        # dyadic fields also try their small inverse levels as marches
        cands = [{**c, "small_march": sm, "small_march_fwd": mf} for sm in SMALL_MARCH_CHOICES
                 for mf in SMALL_MARCH_FWD_CHOICES for c in SINGLE_CANDIDATES]
    for cand in cands:
        set_single(lib, cand)
        arc = waltz_b200.compress_tensor(f, eb, tuned=False)
        tc = _time(torch, lambda: waltz_b200.compress_tensor(f, eb, tuned=False), reps)
        td = _time(torch, lambda: waltz_b200.decompress_tensor(arc, shape, dtype, tuned=False), reps)
        results.append({"knobs": cand, "compress_ms": round(tc, 4), "decompress_ms": round(td, 4)})
    entry = {"class": single_class(shape, itemsize), "workload": f"{dtype} {shape} k^-11/3 REL {rel:g}",
             "measured": results}
    choice = min(results, key=lambda r: r["compress_ms"] + r["decompress_ms"])["knobs"]
    entry["choice"] = dict(choice)
    # every precision-form split where it applies, timed with the chosen
    # knobs (form="auto" takes choose_matrix's pick among them)
    if waltz_b200._matrix_ok(shape, itemsize):
        set_single(lib, choice)
        plain_bytes = int(waltz_b200.compress_tensor(f, eb, tuned=False).numel())
        entry["plain_archive_bytes"] = plain_bytes
        forms = {}
        for form in MATRIX_SPLITS:
            if not waltz_b200._matrix_ok(shape, itemsize, form):
                continue
            arc = waltz_b200.compress_tensor(f, eb, form=form, tuned=False)
            tc = _time(torch, lambda: waltz_b200.compress_tensor(f, eb, form=form, tuned=False), reps)
            td = _time(torch, lambda: waltz_b200.decompress_tensor(arc, shape, dtype, tuned=False), reps)
            forms[form] = {"compress_ms": round(tc, 4), "decompress_ms": round(td, 4),
                           "archive_bytes": int(arc.numel())}
        entry["matrix_forms"] = forms
        entry["choice"]["matrix"] = choose_matrix(entry, itemsize)
    set_single(lib, {})
    return entry


def _tune_batch(torch, lib, fields, label, reps, rel=1e-3):
    import waltz_b200
    bounds = []
    for f in fields:
        lo, hi = waltz_b200.extrema(f)
        bounds.append(rel * (hi - lo))
    shapes = [tuple(f.shape) for f in fields]
    itemsize = fields[0].element_size()
    cap = sum(waltz_b200.compressed_capacity(f.numel(), itemsize) + 16 for f in fields)
    out = torch.empty(cap, dtype=torch.uint8, device=fields[0].device)
    dec = torch.empty(sum(f.numel() for f in fields), dtype=fields[0].dtype, device=fields[0].device)
    results = []
    for cand in BATCH_CANDIDATES:
        lib.waltz_b200_batch_config(cand["mode"], cand["width"])
        set_single(lib, batch_single_knobs(cand))
        arcs = waltz_b200.compress_batch(fields, bounds, out=out, tuned=False)
        tc = _time(torch, lambda: waltz_b200.compress_batch(fields, bounds, out=out, tuned=False), reps)
        td = _time(torch, lambda: waltz_b200.decompress_batch(arcs, shapes, fields[0].dtype, out=dec, tuned=False),
                   reps)
        results.append({"knobs": cand, "compress_ms": round(tc, 4), "decompress_ms": round(td, 4)})
    lib.waltz_b200_batch_config(*[DEFAULT_BATCH[k] for k in ("mode", "width")])
    set_single(lib, {})
    choice = min(results, key=lambda r: r["compress_ms"] + r["decompress_ms"])["knobs"]
    return {"class": batch_class(shapes, itemsize), "workload": label, "measured": results, "choice": dict(choice)}


def tune(quick=False, reps=5, path=TABLE):
    """Measure every candidate on the standard workloads and write the table."""
    import torch
    from . import _lib
    from .synthetic import power_law_field_device, uneven_chunks_device
    lib = _lib.lib()
    entries = []
    singles = [((64, 64, 64), torch.float32), ((256, 256, 256), torch.float32), ((512, 512, 512), torch.float32),
               ((32, 128, 128), torch.float32), ((64, 1024, 1024), torch.float32), ((96, 256, 384), torch.float64)]
    if quick:
        singles = singles[:2] + singles[3:5]
    for shape, dtype in singles:
        t = time.time()
        entries.append(_tune_single(torch, lib, shape, dtype, reps))
        print(f"single {dtype} {shape}: {entries[-1]['choice']} ({time.time() - t:.1f} s)", flush=True)
    batches = [("512 f32 chunks, sides from {32,48,64,96,128} (seed 4), k^-11/3, ranges log-uniform [1e-2,1e3]",
                lambda: uneven_chunks_device(512 if not quick else 128, 4)),
               ("512 f32 chunks 32^3", lambda: [power_law_field_device((32, 32, 32), 100 + i) for i in range(512)]),
               ("64 f32 chunks 128^3", lambda: [power_law_field_device((128, 128, 128), 200 + i) for i in range(64)])]
    for label, make in batches:
        t = time.time()
        fields = [f.contiguous() for f in make()]
        entries.append(_tune_batch(torch, lib, fields, label, reps))
        print(f"batch {label[:40]}: {entries[-1]['choice']} ({time.time() - t:.1f} s)", flush=True)
        del fields
        torch.cuda.empty_cache()
    table = {"device": torch.cuda.get_device_name(), "reps": reps,
             "note": "median CUDA-event times per candidate through the Python API (same call overhead for "
                     "every candidate); choice = least compress + decompress time; matrix = the fastest "
                     "precision-form split (double fields: exact slices only) at least 3 % faster than the "
                     "chosen plain knobs whose archive is at most 2 % larger than the plain one (false: none)",
             "entries": entries}
    Path(path).write_text(json.dumps(table, indent=1) + "\n")
    _cache.pop(str(path), None)
    return table


if __name__ == "__main__":
    import sys
    tune(quick="--quick" in sys.argv, path=Path(sys.argv[sys.argv.index("--out") + 1]) if "--out" in sys.argv else TABLE)
