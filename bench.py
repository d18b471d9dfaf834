"""Benchmark of the Waltz B200 compressor hot path.

Workload (N=1): float32 512x512x512 Gaussian random field with power
spectrum k^-11/3 (unit variance, seed 1), REL 1e-3 bound resolved on the GPU
(eb = 1e-3 * (max - min)), dyadic schedule with 5 levels per axis. A step is
one compress of the field followed by one decompress of its archive; the
metric is the field's bytes per second through that round trip (decimal GB/s),
with compress and decompress throughput and their HBM-roofline fractions
reported beside it. The 512 MiB input and output exceed the 126 MB L2, so no
flush is needed between steps.

N>1 (torchrun): one compressor per GPU on its own copy of the field
(replicas, no collective on the data path); value = all ranks' bytes / max
time over ranks.

`--impl reference` times the reference's own CPU codec (compiled from its
sources into oracle/_ref, AVX2 backend) on the same workload: the field as
one archive, compress + decompress per step. The codec has no threads of its
own, so that is one core; `parallel_blocks` beside it gives its throughput
with the field cut into independent blocks, one per host thread.

Beside the line's own numbers: `cpu_baseline` (the reference CPU codec, one
core, the field as one archive, once) and `gpu_baseline` (the reference's own CUDA library,
built from its sources for sm_100a, on the same field, bound and GPU, with
its archive compared byte for byte with ours); `tc_form` / `tc_form_f64`
compare the plain and precision forms on the float 1024x1024x64 and double
384x256x96 plane-schedule configurations; `batched_form` the batched form on
512 uneven chunks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "comp/decomp GB/s f32 512^3 REL1e-3, plain vs TC form at same bound; % HBM peak"
SHAPE = (512, 512, 512)
REL = 1e-3
SEED = 1


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, line in self.lines:
            if not (t0 - 0.05 <= t <= t1 + 0.05):
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------- GPU arm
def gpu_arm(args, rank, world, local_rank):
    import torch
    import waltz_b200
    from waltz_b200 import _lib
    from waltz_b200.synthetic import power_law_field_device

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = _lib.lib()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    shape = tuple(args.shape)
    from waltz_b200 import autotune
    knobs = autotune.apply_single(lib, shape, 4)  # committed tuning table (never changes the bytes)
    field = power_law_field_device(shape, SEED, device=dev).contiguous()
    n = field.numel()
    nbytes = n * 4
    lo, hi = waltz_b200.extrema(field)
    eb = REL * (hi - lo)
    cap = waltz_b200.compressed_capacity(n, 4)
    archive = torch.empty(cap, dtype=torch.uint8, device=dev)
    out = torch.empty_like(field)
    nz, ny, nx = shape
    written = C.c_size_t()

    def compress():
        _lib.checked(lib.waltz_b200_compress(C.c_void_p(field.data_ptr()), 4, nx, ny, nz, eb,
                                             C.c_void_p(archive.data_ptr()), cap, C.byref(written), sp))
        return written.value

    def decompress(size):
        _lib.checked(lib.waltz_b200_decompress(C.c_void_p(archive.data_ptr()), size, 4, nx, ny, nz,
                                               C.c_void_p(out.data_ptr()), nbytes, sp))

    # correctness of the measured configuration (untimed)
    size = compress()
    decompress(size)
    max_err = float((out.double() - field.double()).abs().max())
    assert max_err <= eb, f"bound violated: {max_err} > {eb}"
    first = archive[:size].clone()
    header = first[:32].cpu().numpy().tobytes()
    n_repairs, n_qout = int.from_bytes(header[24:28], "little"), int.from_bytes(header[28:32], "little")

    for _ in range(args.warmup):
        decompress(compress())

    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    dist_barrier(world)
    torch.cuda.synchronize()
    launches0 = lib.waltz_b200_launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    t_wall0 = time.time()
    ev[0].record(stream)
    for k in range(args.steps):
        size = compress()
        ev[2 * k + 1].record(stream)
        decompress(size)
        ev[2 * k + 2].record(stream)
    torch.cuda.synchronize()
    t_wall1 = time.time()
    launches = lib.waltz_b200_launch_count() - launches0
    dist_barrier(world)
    sampler.stop()
    comp_ms = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)]
    dec_ms = [ev[2 * k + 1].elapsed_time(ev[2 * k + 2]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    total_ms = dist_max(total_ms, world)
    assert torch.equal(archive[:size], first), "archive changed between steps"

    # ---- per-kernel stage timing (separate, untimed pass)
    lib.waltz_b200_profile(1)
    stages = {}
    for _ in range(3):
        size = compress()
        times = (C.c_double * 16)()
        names = (C.c_char_p * 16)()
        cnt = lib.waltz_b200_stage_times(times, names, 16)
        for i in range(cnt):
            stages.setdefault("compress:" + names[i].decode(), []).append(times[i])
        decompress(size)
        cnt = lib.waltz_b200_stage_times(times, names, 16)
        for i in range(cnt):
            stages.setdefault("decompress:" + names[i].decode(), []).append(times[i])
    lib.waltz_b200_profile(0)
    stage_ms = {k: statistics.median(v) for k, v in stages.items()}

    # ---- end to end through the public API with host buffers. Every step
    # copies its field in from pinned host memory, compresses, copies the
    # archive out to the host, copies it back in, decompresses and copies the
    # field out. Serial: one step at a time on one stream. Streamed (the e2e
    # value): two buffer sets, uploads / kernels / downloads on three streams,
    # so a step's copies overlap its neighbours' kernels and both PCIe
    # directions run at once, as a user streaming fields through the codec
    # would run it.
    host_in = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    host_in.copy_(field.cpu())
    host_arch = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
    host_out = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    e2e_ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e2e = []
    for k in range(max(2, min(args.steps, 5)) + 1):
        dist_barrier(world)
        torch.cuda.synchronize()
        e2e_ev[0].record(stream)
        field.copy_(host_in, non_blocking=True)
        s = compress()
        host_arch[:s].copy_(archive[:s], non_blocking=True)
        e2e_ev[1].record(stream)
        archive[:s].copy_(host_arch[:s], non_blocking=True)
        decompress(s)
        host_out.copy_(out, non_blocking=True)
        e2e_ev[2].record(stream)
        torch.cuda.synchronize()
        if k:  # first pass warms the pinned paths
            e2e.append((e2e_ev[0].elapsed_time(e2e_ev[1]), e2e_ev[1].elapsed_time(e2e_ev[2])))
    e2e_c = statistics.median(x[0] for x in e2e)
    e2e_d = statistics.median(x[1] for x in e2e)
    e2e_serial = dist_max(e2e_c + e2e_d, world)
    del host_arch, host_out

    # streamed: a three-deep software pipeline over three buffer sets. Per
    # step k the host issues the upload of field k+1, compresses field k,
    # sends archive k down and back up on streams of their own, decompresses
    # archive k-1 and sends its output down. Field uploads and archive
    # uploads run on separate streams (one does not queue behind the other);
    # downloads on a third; events order every buffer's reuse. The library's
    # calls are synchronous on their stream, so the copies already issued
    # keep both PCIe directions busy while the host waits in a call.
    up, up2, comp, down = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    NSLOT = 3
    slots = []
    for _ in range(NSLOT):
        slots.append({"field": torch.empty_like(field), "out": torch.empty_like(field),
                      "arch": torch.empty(cap, dtype=torch.uint8, device=dev),
                      "harch": torch.empty(cap, dtype=torch.uint8, pin_memory=True),
                      "hout": torch.empty(shape, dtype=torch.float32, pin_memory=True),
                      "size": 0,
                      **{ev: torch.cuda.Event() for ev in ("uploaded", "read", "arch_down", "arch_up", "decoded",
                                                            "downloaded")}})

    def comp_on(sl):
        w = C.c_size_t()
        _lib.checked(lib.waltz_b200_compress(C.c_void_p(sl["field"].data_ptr()), 4, nx, ny, nz, eb,
                                             C.c_void_p(sl["arch"].data_ptr()), cap, C.byref(w),
                                             C.c_void_p(comp.cuda_stream)))
        return w.value

    def dec_on(sl, size):
        _lib.checked(lib.waltz_b200_decompress(C.c_void_p(sl["arch"].data_ptr()), size, 4, nx, ny, nz,
                                               C.c_void_p(sl["out"].data_ptr()), nbytes, C.c_void_p(comp.cuda_stream)))

    def upload(sl):
        up.wait_event(sl["read"])  # the compress that read this buffer last is done
        with torch.cuda.stream(up):
            sl["field"].copy_(host_in, non_blocking=True)
        sl["uploaded"].record(up)

    def streamed(steps_e2e):
        dist_barrier(world)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(comp)
        for st in (up, up2, down):
            st.wait_event(start)
        for sl in slots:
            for ev in ("read", "arch_up", "downloaded"):
                sl[ev].record(comp)
        upload(slots[0])
        for k in range(steps_e2e + 1):
            if k < steps_e2e:
                sl = slots[k % NSLOT]
                if k + 1 < steps_e2e:  # the next field crosses PCIe during this step
                    upload(slots[(k + 1) % NSLOT])
                comp.wait_event(sl["uploaded"])
                comp.wait_event(sl["downloaded"])  # the output this buffer set held last has left
                sl["size"] = size = comp_on(sl)
                sl["read"].record(comp)
                down.wait_event(sl["read"])
                down.wait_event(sl["arch_up"])  # the host archive buffer is free
                with torch.cuda.stream(down):
                    sl["harch"][:size].copy_(sl["arch"][:size], non_blocking=True)
                sl["arch_down"].record(down)
                up2.wait_event(sl["arch_down"])
                with torch.cuda.stream(up2):
                    sl["arch"][:size].copy_(sl["harch"][:size], non_blocking=True)
                sl["arch_up"].record(up2)
            if k >= 1:  # the previous step's archive is back: decode it
                pl = slots[(k - 1) % NSLOT]
                comp.wait_event(pl["arch_up"])
                dec_on(pl, pl["size"])
                pl["decoded"].record(comp)
                down.wait_event(pl["decoded"])
                with torch.cuda.stream(down):
                    pl["hout"].copy_(pl["out"], non_blocking=True)
                pl["downloaded"].record(down)
        for st in (up, up2, down):
            comp.wait_stream(st)
        end.record(comp)
        torch.cuda.synchronize()
        return start.elapsed_time(end)

    steps_e2e = max(6, min(args.steps, 12))
    streamed(NSLOT)  # warm the pinned paths of every buffer set
    e2e_ms = dist_max(streamed(steps_e2e), world) / steps_e2e
    worst = max(float((sl["hout"].double() - host_in.double()).abs().max()) for sl in slots)
    assert worst <= eb, f"streamed end-to-end result violates the bound: {worst} > {eb}"

    # the copy ceiling of that pipeline: a field's bytes up and a field's
    # bytes down at the same time, no kernels (per-direction GB/s, best of 3)
    def both_ways(reps=3):
        best = None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(comp)
            up.wait_event(t0)
            down.wait_event(t0)
            with torch.cuda.stream(up):
                slots[0]["field"].copy_(host_in, non_blocking=True)
            with torch.cuda.stream(down):
                slots[1]["hout"].copy_(slots[1]["out"], non_blocking=True)
            comp.wait_stream(up)
            comp.wait_stream(down)
            t1.record(comp)
            torch.cuda.synchronize()
            ms = t0.elapsed_time(t1)
            best = ms if best is None else min(best, ms)
        return nbytes / (best / 1e3) / 1e9

    pcie_gbs = both_ways()
    del slots

    hbm, peak_kind = peaks()
    t_c = statistics.median(comp_ms) / 1e3
    t_d = statistics.median(dec_ms) / 1e3
    a_bytes = size
    step_ms = total_ms / args.steps
    value = world * nbytes / (step_ms / 1e3) / 1e9
    algo = algorithmic_bytes(n, 4, a_bytes, fused="compress:quantize" not in stage_ms)
    dom, dom_ms = max(((k, v) for k, v in stage_ms.items() if k in algo), key=lambda kv: kv[1])
    achieved = algo[dom] / (dom_ms / 1e3) / 1e9
    result = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(step_ms, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded k^-11/3 Gaussian random field (stand-in for the reference's simulation fields)",
        "config": {"workload": "f32 %dx%dx%d (z,y,x) k^-11/3 GRF seed 1, REL 1e-3 (eb=%.6g), "
                               "step = compress + decompress" % (*shape, eb),
                   "global_batch": world, "seq_len": None, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (512 MiB field)", "archive_bytes": a_bytes,
                   "compression_ratio": round(nbytes / a_bytes, 4), "max_abs_error": max_err, "abs_bound": eb,
                   "repair_records": n_repairs, "q_outliers": n_qout, "tuning": knobs},
        "compress_gbs": round(nbytes / t_c / 1e9, 3),
        "decompress_gbs": round(nbytes / t_d / 1e9, 3),
        "compress_hbm_frac": round((nbytes + a_bytes) / t_c / 1e9 / hbm, 4),
        "decompress_hbm_frac": round((nbytes + a_bytes) / t_d / 1e9 / hbm, 4),
        "stage_ms": {k: round(v, 4) for k, v in sorted(stage_ms.items())},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 2), "peak": hbm,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "algorithmic_bytes": algo[dom], "traffic": None},
        "e2e": {"value": round(world * nbytes / (e2e_ms / 1e3) / 1e9, 3), "unit": "GB/s",
                "h2d_bytes_per_step": nbytes + a_bytes, "d2h_bytes_per_step": a_bytes + nbytes,
                "form": f"streamed: {steps_e2e} steps, three-deep pipeline; field uploads, archive round trips, "
                        "kernels and downloads on their own streams, three buffer sets",
                "ms_per_step": round(e2e_ms, 4),
                # a step's copies alone at the measured two-way rate: the ceiling of `value`
                "pcie_both_ways_gbs": round(pcie_gbs, 3),
                "copy_ceiling": round(world * nbytes / ((nbytes + a_bytes) / (pcie_gbs * 1e9)) / 1e9, 3),
                "serial": {"value": round(world * nbytes / (e2e_serial / 1e3) / 1e9, 3), "compress_ms": round(e2e_c, 4),
                           "decompress_ms": round(e2e_d, 4)}},
        "gpu_launches": int(launches),
        "clocks": sampler.summary(t_wall0, t_wall1),
    }
    if shape == SHAPE and dom in TRAFFIC_512:
        result["roofline"]["traffic"] = TRAFFIC_512[dom]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        host_field = field.cpu().numpy()
        result["cpu_baseline"] = cpu_baseline(host_field, eb, first)
        result["archive_identical_to_cpu"] = result["cpu_baseline"].get("archive_identical_to_ours")
    if world == 1:
        rel2 = 1e-4
        result[f"rel_{rel2:g}"] = bound_entry(lib, field, rel2 * (hi - lo), min(args.steps, 10), hbm,
                                              host_field if rank == 0 and not args.no_cpu_baseline else None)
    if rank == 0 and world == 1 and not args.no_gpu_baseline:
        result["gpu_baseline"] = gpu_baseline(field, eb, archive[:a_bytes], min(args.steps, 10))
    if not args.no_tc_form and world == 1:
        del field, out, archive, host_in
        torch.cuda.empty_cache()
        result["tc_form"] = tc_form_comparison(dev, lib, args.steps, tuple(args.tc_shape),
                                               ref_gpu=rank == 0 and not args.no_gpu_baseline)
        torch.cuda.empty_cache()
        result["tc_form_f64"] = tc_form_f64(dev, lib, args.steps, ref_gpu=rank == 0 and not args.no_gpu_baseline)
    if not args.no_batch and world > 1:
        torch.cuda.empty_cache()
        result["batched_form_sharded"] = batch_sharded(dev, lib, args.steps, rank, world)
    if not args.no_batch and world == 1:
        torch.cuda.empty_cache()
        result["batched_form"] = batch_comparison(dev, lib, args.steps,
                                                  cpu=rank == 0 and not args.no_cpu_baseline,
                                                  ref_gpu=rank == 0 and not args.no_gpu_baseline)
    return result


def cpu_identical(host_field, eb, ours):
    """Whether our archive equals the reference CPU codec's (oracle/_ref, AVX2,
    whose bytes equal its scalar backend's) for the same field and bound."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    expect = O.RefCodec(O.AVX2).compress(host_field, eb)
    return len(expect) == ours.numel() and expect == ours.cpu().numpy().tobytes()


def bound_entry(lib, field, eb, steps, hbm, host_field=None):
    """Compress and decompress throughput of the device-resident field at
    another bound: CUDA events around each call, median over `steps` after two
    warm-up steps; the archive compared with the reference CPU codec's when
    `host_field` is given."""
    import torch
    import waltz_b200
    from waltz_b200 import _lib
    n = field.numel()
    nbytes = n * field.element_size()
    nz, ny, nx = field.shape
    cap = waltz_b200.compressed_capacity(n, 4)
    arch = torch.empty(cap, dtype=torch.uint8, device=field.device)
    out = torch.empty_like(field)
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    w = C.c_size_t()
    tc, td = [], []
    for it in range(2 + steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        _lib.checked(lib.waltz_b200_compress(C.c_void_p(field.data_ptr()), 4, nx, ny, nz, eb,
                                             C.c_void_p(arch.data_ptr()), cap, C.byref(w), sp))
        e[1].record()
        _lib.checked(lib.waltz_b200_decompress(C.c_void_p(arch.data_ptr()), w.value, 4, nx, ny, nz,
                                               C.c_void_p(out.data_ptr()), nbytes, sp))
        e[2].record()
        torch.cuda.synchronize()
        if it >= 2:
            tc.append(e[0].elapsed_time(e[1]))
            td.append(e[1].elapsed_time(e[2]))
    a = w.value
    t_c, t_d = statistics.median(tc) / 1e3, statistics.median(td) / 1e3
    header = arch[:32].cpu().numpy().tobytes()
    entry = {"abs_bound": eb, "archive_bytes": a, "compression_ratio": round(nbytes / a, 4),
             "compress_gbs": round(nbytes / t_c / 1e9, 3), "decompress_gbs": round(nbytes / t_d / 1e9, 3),
             "compress_hbm_frac": round((nbytes + a) / t_c / 1e9 / hbm, 4),
             "decompress_hbm_frac": round((nbytes + a) / t_d / 1e9 / hbm, 4),
             "value": round(nbytes / (t_c + t_d) / 1e9, 3),
             "repair_records": int.from_bytes(header[24:28], "little"),
             "q_outliers": int.from_bytes(header[28:32], "little"),
             "max_abs_error": float((out.double() - field.double()).abs().max())}
    if host_field is not None:
        entry["archive_identical_to_cpu"] = cpu_identical(host_field, eb, arch[:a])
    del arch, out
    return entry


# the precision form's tensor-core splits (WALTZ_B200_FORM_MATRIX*)
SPLIT_FORMS = (("matrix_tf32x3", 1), ("matrix_bf16x3", 2), ("matrix_exact", 3))


def _form_entries(dev, lib, f, eb, steps, ref_gpu):
    """Plain lifting and every split of the precision form on one
    device-resident field at one absolute bound: compress / decompress GB/s
    (median of `steps` after one warm-up), ratio, repair records, worst error,
    and each split's ratio change against the plain form; beside them the
    reference's own CUDA library (the plain form's bytes)."""
    import torch
    import waltz_b200
    from waltz_b200 import _lib
    nz, ny, nx = f.shape
    width = f.element_size()
    n = f.numel()
    nbytes = n * width
    cap = waltz_b200.compressed_capacity(n, width)
    arch = torch.empty(cap, dtype=torch.uint8, device=dev)
    out = torch.empty_like(f)
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    written = C.c_size_t()
    entry = {}
    plain_arch = None
    for form, code in (("plain", 0),) + SPLIT_FORMS:
        def comp():
            _lib.checked(lib.waltz_b200_compress_form(C.c_void_p(f.data_ptr()), width, nx, ny, nz, eb, code,
                                                      C.c_void_p(arch.data_ptr()), cap, C.byref(written), sp))
            return written.value

        def dec(size):
            _lib.checked(lib.waltz_b200_decompress(C.c_void_p(arch.data_ptr()), size, width, nx, ny, nz,
                                                   C.c_void_p(out.data_ptr()), nbytes, sp))
        try:
            size = comp()
        except _lib.WaltzError as e:  # the form cannot serve this field at this bound
            entry[form] = {"error": str(e), "abs_bound": eb}
            continue
        dec(size)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        tc, td = [], []
        for _ in range(max(1, steps)):
            ev[0].record()
            size = comp()
            ev[1].record()
            dec(size)
            ev[2].record()
            torch.cuda.synchronize()
            tc.append(ev[0].elapsed_time(ev[1]))
            td.append(ev[1].elapsed_time(ev[2]))
        # per-stage device times of one more compress + decompress (profiling on)
        lib.waltz_b200_profile(1)
        stage = {}
        times, names = (C.c_double * 16)(), (C.c_char_p * 16)()
        size = comp()
        for i in range(lib.waltz_b200_stage_times(times, names, 16)):
            stage["compress:" + names[i].decode()] = round(times[i], 4)
        dec(size)
        for i in range(lib.waltz_b200_stage_times(times, names, 16)):
            stage["decompress:" + names[i].decode()] = round(times[i], 4)
        lib.waltz_b200_profile(0)
        header = arch[:32].cpu().numpy().tobytes()
        err = float((out.double() - f.double()).abs().max())
        assert err <= eb, f"{form} form violates the bound: {err} > {eb}"
        entry[form] = {"compress_gbs": round(nbytes / (statistics.median(tc) / 1e3) / 1e9, 3),
                       "decompress_gbs": round(nbytes / (statistics.median(td) / 1e3) / 1e9, 3),
                       "compression_ratio": round(nbytes / size, 4),
                       "repair_records": int.from_bytes(header[24:28], "little"),
                       "max_abs_error": err, "abs_bound": eb, "stage_ms": stage}
        if form == "plain":
            plain_arch = arch[:size].clone()
    if "compression_ratio" in entry["plain"]:
        entry["ratio_change"] = {form: round(entry[form]["compression_ratio"] / entry["plain"]["compression_ratio"] - 1,
                                             5)
                                 for form, _ in SPLIT_FORMS if "compression_ratio" in entry[form]}
    if ref_gpu and plain_arch is not None:
        entry["reference_gpu"] = gpu_baseline(f, eb, plain_arch, max(1, steps))
    del plain_arch, arch, out
    return entry


def _z_coefficient_error(dev, lib, f):
    """Largest error of the tensor-core Z stage, in every split, against the
    float64 lifting on up to 16384 columns of the field (absolute, and
    relative to the largest coefficient of each column)."""
    import torch
    from waltz_b200 import _lib
    nz, ny, nx = f.shape
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    cols = min(16384, nx * ny)
    x = f.reshape(nz, -1)[:, :cols].contiguous()
    eye = torch.eye(nz, dtype=torch.float64, device=dev).reshape(nz, nz, 1, 1)
    m = torch.empty(nz, nz, dtype=torch.float64, device=dev)
    for k in range(nz):
        e = eye[:, k].contiguous()
        _lib.checked(lib.waltz_b200_transform(C.c_void_p(e.data_ptr()), 8, 1, 1, nz, 0, sp))
        m[:, k] = e.reshape(nz)
    ref = m @ x.double()
    report = {"columns": cols}
    for form, code in SPLIT_FORMS:
        tcx = x.clone()
        rc = lib.waltz_b200_zmatrix_split(C.c_void_p(tcx.data_ptr()), f.element_size(), cols, 1, nz, 0, code, sp)
        if rc != 0:
            report[form] = {"error": _lib.last_error()}
            continue
        diff = (tcx.double() - ref).abs()
        report[form] = {"max_abs": float(diff.max()),
                        "max_rel_to_column_max": float((diff.max(0).values /
                                                        ref.abs().max(0).values.clamp_min(1e-30)).max())}
    return report


def tc_form_comparison(dev, lib, steps, shape=(64, 1024, 1024), ref_gpu=True):
    """Plain lifting against every split of the precision form (tensor-core Z
    stage) on the tensor-core configuration: float32 1024x1024x64 (z=64) k^-11/3 random field
    (seed 3) with 1 % salt spikes of magnitude 50, REL 1e-3 and 1e-5; device
    resident, CUDA events, median of `steps` after one warm-up; beside them the
    reference's own CUDA library (its default profile, the plain form's bytes)
    on the same field and bound. Also the Z-stage coefficient error of the
    tensor-core matrix against the float64 lifting transform on 16384 columns
    of the field."""
    import torch
    import waltz_b200
    from waltz_b200 import autotune
    from waltz_b200.synthetic import spiky_field_device
    autotune.apply_single(lib, shape, 4)  # this field's class in the tuning table (never changes the bytes)
    f = spiky_field_device(shape, 3, device=dev)
    lo, hi = waltz_b200.extrema(f)
    report = {"workload": "f32 %dx%dx%d (z,y,x) k^-11/3 GRF seed 3 + 1%% spikes of 50, plane schedule" % shape}
    for rel in (1e-3, 1e-5):
        report[f"rel_{rel:g}"] = _form_entries(dev, lib, f, rel * (hi - lo), steps, ref_gpu)
    report["z_coefficient_error_vs_float64"] = _z_coefficient_error(dev, lib, f)
    return report


def tc_form_f64(dev, lib, steps, shape=(96, 256, 384), ref_gpu=True):
    """The same comparison on the double configuration: float64 384x256x96
    (z=96) k^-5/3 random field (seed 2) plus a front 10*tanh((z-48)/2) along
    z, ABS 1e-4, 1e-5 and 1e-6, every split of the precision form: TF32x3 and
    BF16x3 are fp32-accurate, the exact bf16 slices double-accurate; the
    quantisation and repair decisions stay in double, and the repair pass
    restores the bound."""
    import torch
    from waltz_b200 import autotune
    from waltz_b200.synthetic import front_field
    autotune.apply_single(lib, shape, 8)
    f = torch.from_numpy(front_field(shape, 2)).to(dev).contiguous()
    report = {"workload": "f64 %dx%dx%d (z,y,x) k^-5/3 GRF seed 2 + 10*tanh((z-48)/2), plane schedule" % shape}
    # at ABS 1e-6 this field's coefficients exceed 65535 quanta so often that
    # the q-outlier list passes the portable side-channel cap (2^20 records for
    # fields over 2^20 samples) in either form, as in the reference; the entry
    # records the refusal, the looser bounds measure both forms
    for eb in (1e-4, 1e-5, 1e-6):
        report[f"abs_{eb:g}"] = _form_entries(dev, lib, f, eb, steps, ref_gpu)
    report["z_coefficient_error_vs_float64"] = _z_coefficient_error(dev, lib, f)
    return report


def batch_comparison(dev, lib, steps, count=512, cpu=False, ref_gpu=False):
    """Batched form against one call per chunk on the uneven-chunk workload:
    512 float32 chunks, per-axis sides drawn from {32,48,64,96,128} (seed 4),
    k^-11/3 fields each rescaled to a range drawn log-uniformly in [1e-2,1e3],
    REL 1e-3 per chunk. Batched: waltz_b200_compress_batch (one graph) and
    waltz_b200_decompress_batch into one preallocated tensor (one graph,
    archives read from one staging buffer). Per-chunk: waltz_b200_compress /
    waltz_b200_decompress once per chunk. Device-resident; CUDA events per
    batch; latency percentiles over the timed batches after warm-up (the
    first batched call captures the graphs)."""
    import torch
    import waltz_b200
    from waltz_b200 import _lib
    from waltz_b200.synthetic import uneven_chunks_device
    fields = uneven_chunks_device(count, 4, device=dev)
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    sizes = [f.numel() for f in fields]
    nbytes = 4 * sum(sizes)
    bounds = []
    for f in fields:
        lo, hi = waltz_b200.extrema(f)
        bounds.append(REL * (hi - lo))
    caps = [waltz_b200.compressed_capacity(k, 4) for k in sizes]
    offs = [0]
    for c in caps:
        offs.append(offs[-1] + (c + 255) // 256 * 256)
    arch = torch.empty(offs[-1], dtype=torch.uint8, device=dev)
    items = (_lib.Chunk * count)()
    for i, f in enumerate(fields):
        nz, ny, nx = f.shape
        items[i] = _lib.Chunk(f.data_ptr(), nx, ny, nz, bounds[i], arch.data_ptr() + offs[i], caps[i])
    written = (C.c_uint64 * count)()
    out = torch.empty(sum(sizes), dtype=torch.float32, device=dev)
    outs, at = [], 0
    for k in sizes:
        outs.append(out[at:at + k])
        at += k

    def comp_batch():
        _lib.checked(lib.waltz_b200_compress_batch(items, count, 4, written, sp))

    dec_items = (_lib.Archive * count)()

    def dec_batch():
        _lib.checked(lib.waltz_b200_decompress_batch(dec_items, count, 4, sp))

    one = C.c_size_t()

    def comp_each():
        for i, f in enumerate(fields):
            nz, ny, nx = f.shape
            _lib.checked(lib.waltz_b200_compress(C.c_void_p(f.data_ptr()), 4, nx, ny, nz, bounds[i],
                                                 C.c_void_p(arch.data_ptr() + offs[i]), caps[i], C.byref(one), sp))

    def dec_each():
        for i, f in enumerate(fields):
            nz, ny, nx = f.shape
            _lib.checked(lib.waltz_b200_decompress(C.c_void_p(arch.data_ptr() + offs[i]), written[i], 4, nx, ny, nz,
                                                   C.c_void_p(outs[i].data_ptr()), 4 * sizes[i], sp))

    def timed(fn, reps):
        ms = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    from waltz_b200 import autotune
    batch_knobs = autotune.apply_batch(lib, [tuple(f.shape) for f in fields], 4)
    comp_batch()
    first = [bytes(arch[offs[i]:offs[i] + written[i]].cpu().numpy()) for i in range(0, count, 37)]
    for i, f in enumerate(fields):
        nz, ny, nx = f.shape
        dec_items[i] = _lib.Archive(arch.data_ptr() + offs[i], written[i], None, nx, ny, nz, outs[i].data_ptr(),
                                    4 * sizes[i])
    dec_batch()
    worst = max(float((o.view(f.shape).double() - f.double()).abs().max()) / eb
                for o, f, eb in zip(outs, fields, bounds))
    assert worst <= 1.0, f"bound violated in the batch: {worst}"
    archive_bytes = sum(written)
    reps = max(steps, 20)
    for _ in range(3):
        comp_batch()
        dec_batch()
    cb = timed(comp_batch, reps)
    db = timed(dec_batch, reps)
    # the one-call-per-chunk path with the library defaults
    lib.waltz_b200_set_option(autotune.OPT_STAGE_KERNELS, 1)
    lib.waltz_b200_set_option(autotune.OPT_ZMARCH_PLANES, 0)
    ce = timed(comp_each, max(3, steps // 4))
    de = timed(dec_each, max(3, steps // 4))
    # per-chunk archives equal the batched ones
    for j, i in enumerate(range(0, count, 37)):
        assert bytes(arch[offs[i]:offs[i] + written[i]].cpu().numpy()) == first[j], "batched archive differs"

    def stats(ms):
        ms = sorted(ms)
        med = statistics.median(ms)
        return {"chunks_per_s": round(count / (med / 1e3), 1), "gbs": round(nbytes / (med / 1e3) / 1e9, 3),
                "p50_ms": round(med, 4), "p99_ms": round(ms[min(len(ms) - 1, int(0.99 * len(ms)))], 4),
                "batches": len(ms)}
    report = {
        "workload": f"{count} f32 chunks, sides per axis from {{32,48,64,96,128}} (seed 4), k^-11/3 fields, "
                    "ranges log-uniform in [1e-2,1e3], REL 1e-3 per chunk",
        "samples": sum(sizes), "bytes": nbytes, "archive_bytes": archive_bytes,
        "compression_ratio": round(nbytes / archive_bytes, 4), "max_err_over_bound": round(worst, 6),
        "batch_tuning": batch_knobs,
        "compress": {"batched": stats(cb), "per_chunk": stats(ce)},
        "decompress": {"batched": stats(db), "per_chunk": stats(de)},
    }
    for k in ("compress", "decompress"):
        report[k]["speedup"] = round(report[k]["batched"]["gbs"] / report[k]["per_chunk"]["gbs"], 3)
    # compress + decompress throughput of the batched form, as the CPU line measures it
    report["batched_gbs"] = round(nbytes / ((statistics.median(cb) + statistics.median(db)) / 1e3) / 1e9, 3)
    if cpu:
        report["cpu_baseline"] = cpu_batch_baseline([f.cpu().numpy() for f in fields], bounds)
    if ref_gpu:
        report["gpu_baseline"] = gpu_batch_baseline(fields, bounds, arch, offs, written)
    return report


def gpu_batch_baseline(fields, bounds, ours, offs, written, reps=2):
    """The reference's own CUDA library over the same chunk list on the same
    GPU: it has no batched compressor, so one d_compress and one d_decompress
    per chunk (its public API), device-resident, CUDA events around the whole
    list; every archive compared byte for byte with ours."""
    import torch
    from oracle import oracle as O
    if not O.refgpu_available():
        return {"unavailable": "reference CUDA library not built (make -C oracle refgpu)"}
    lib = O.refgpu_lib()
    stream = torch.cuda.current_stream().cuda_stream
    caps = [lib.refgpu_capacity(f.numel(), 4) for f in fields]
    arch = torch.empty(max(caps), dtype=torch.uint8, device=fields[0].device)
    srcs = [f.clone() for f in fields]  # the reference takes mutable input pointers
    out = torch.empty(max(f.numel() for f in fields), dtype=torch.float32, device=fields[0].device)
    identical = True
    for i, f in enumerate(srcs):
        size = O.refgpu_compress(f.data_ptr(), 4, tuple(f.shape), bounds[i], arch.data_ptr(), stream)
        torch.cuda.synchronize()
        identical &= size == written[i] and bool(torch.equal(arch[:size], ours[offs[i]:offs[i] + size]))
    cmp_ms, dec_ms = [], []
    nbytes = 4 * sum(f.numel() for f in fields)
    for _ in range(reps):
        tc = td = 0.0
        for i, f in enumerate(srcs):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            O.refgpu_compress(f.data_ptr(), 4, tuple(f.shape), bounds[i], arch.data_ptr(), stream)
            e[1].record()
            O.refgpu_decompress(arch.data_ptr(), 4, tuple(f.shape), out.data_ptr(), stream)
            e[2].record()
            torch.cuda.synchronize()
            tc += e[0].elapsed_time(e[1])
            td += e[1].elapsed_time(e[2])
        cmp_ms.append(tc)
        dec_ms.append(td)
    t_c, t_d = min(cmp_ms), min(dec_ms)
    del srcs, arch, out
    return {"value": round(nbytes / ((t_c + t_d) / 1e3) / 1e9, 3), "unit": "GB/s",
            "compress_gbs": round(nbytes / (t_c / 1e3) / 1e9, 3),
            "decompress_gbs": round(nbytes / (t_d / 1e3) / 1e9, 3),
            "chunks_per_s": round(len(fields) / ((t_c + t_d) / 1e3), 1),
            "archives_identical_to_ours": identical, "kind": "reference CUDA library, same GPU, one call per chunk",
            "sample": f"all {len(fields)} chunks, best of {reps} passes"}


def batch_sharded(dev, lib, steps, rank, world, count=512):
    """The uneven-chunk batch shared across the ranks (one GPU each): every
    rank builds the same chunk list, takes its share (balanced by bytes,
    waltz_b200.shard.partition) and runs batched compress + decompress of it;
    no data-path collective, only the archive sizes are exchanged once (the
    metadata a shared container needs). Time per step = max over ranks;
    value = the whole batch's bytes / that time (the batch is fixed as the
    ranks grow: strong scaling)."""
    import torch
    import waltz_b200
    from waltz_b200 import autotune, shard
    from waltz_b200.synthetic import uneven_chunks_device
    fields = uneven_chunks_device(count, 4, device=dev)
    sizes = [f.numel() * 4 for f in fields]
    mine = shard.partition(sizes, world)[rank]
    local = [fields[i].contiguous() for i in mine]
    del fields
    bounds = []
    for f in local:
        lo, hi = waltz_b200.extrema(f)
        bounds.append(REL * (hi - lo))
    shapes = [tuple(f.shape) for f in local]
    cap = sum(waltz_b200.compressed_capacity(f.numel(), 4) + 256 for f in local)
    arch_buf = torch.empty(max(cap, 1), dtype=torch.uint8, device=dev)
    out = torch.empty(max(sum(f.numel() for f in local), 1), dtype=torch.float32, device=dev)
    autotune.apply_batch(lib, shapes, 4)
    arcs = []

    def step():
        nonlocal arcs
        if local:
            arcs = waltz_b200.compress_batch(local, bounds, out=arch_buf)
            waltz_b200.decompress_batch(arcs, shapes, torch.float32, out=out)
    for _ in range(2):
        step()
    ms = []
    for _ in range(max(3, steps)):
        dist_barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        ms.append(dist_max(e0.elapsed_time(e1), world))
    sizes_all, _ = shard.exchange_sizes({i: a.numel() for i, a in zip(mine, arcs)}) if world > 1 else (
        {i: a.numel() for i, a in zip(mine, arcs)}, None)
    t = statistics.median(ms)
    loads = [sum(sizes[i] for i in share) for share in shard.partition(sizes, world)]
    return {"workload": f"{count} f32 chunks, sides per axis from {{32,48,64,96,128}} (seed 4), REL 1e-3 per chunk, "
                        f"shared across {world} ranks by bytes",
            "value": round(sum(sizes) / (t / 1e3) / 1e9, 3), "unit": "GB/s", "ms_per_step": round(t, 4),
            "scaling": "strong", "ranks": world, "chunks_this_rank": len(mine),
            "max_rank_bytes_over_mean": round(max(loads) / (sum(loads) / world), 4),
            "archive_bytes": int(sum(sizes_all.values())), "chunks_compressed": len(sizes_all)}


def batch_only(dev, lib, args, count=512):
    """The batched form alone on the uneven-chunk workload: `warmup` + `steps`
    batched compress + decompress calls (the first captures the graphs)."""
    import torch
    import waltz_b200
    from waltz_b200 import autotune
    from waltz_b200.synthetic import uneven_chunks_device
    fields = uneven_chunks_device(count, 4, device=dev)
    bounds = []
    for f in fields:
        lo, hi = waltz_b200.extrema(f)
        bounds.append(REL * (hi - lo))
    shapes = [tuple(f.shape) for f in fields]
    out = torch.empty(sum(waltz_b200.compressed_capacity(f.numel(), 4) + 16 for f in fields), dtype=torch.uint8,
                      device=dev)
    dec = torch.empty(sum(f.numel() for f in fields), dtype=torch.float32, device=dev)
    if args.batch_config:
        parts = [int(v) for v in args.batch_config.split(":")]
        knobs = {"mode": parts[0], "width": parts[1], "stage_kernels": parts[2] if len(parts) > 2 else 1,
                 "zmarch": parts[3] if len(parts) > 3 else 0}
    else:
        knobs = autotune.lookup(autotune.batch_class(shapes, 4))
    lib.waltz_b200_batch_config(knobs["mode"], knobs["width"])
    autotune.set_single(lib, autotune.batch_single_knobs(knobs))
    ms = []
    for k in range(args.warmup + max(1, args.steps)):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        arcs = waltz_b200.compress_batch(fields, bounds, out=out, tuned=False)
        waltz_b200.decompress_batch(arcs, shapes, torch.float32, out=dec, tuned=False)
        b.record()
        torch.cuda.synchronize()
        if k >= args.warmup:
            ms.append(a.elapsed_time(b))
    nbytes = 4 * sum(f.numel() for f in fields)
    return {"workload": f"{count} uneven f32 chunks (seed 4), REL 1e-3, batched compress + decompress",
            "knobs": knobs, "ms_per_step": round(statistics.median(ms), 4),
            "gbs": round(nbytes / (statistics.median(ms) / 1e3) / 1e9, 3)}


# DRAM bytes (read + write) per launch of the finest-level kernels on this
# workload (f32 512^3, REL 1e-3): dram__bytes_read.sum + dram__bytes_write.sum
# of one ncu capture of each kernel's first launch at 512^3
# (profiles/dram_traffic_f32_512cubed_rel1e-3.md). A run on another shape
# reports no traffic.
TRAFFIC_512 = {
    "compress:fwd_l0": 1045993984,
    "compress:wzp_encode": 1110756608,
    "compress:inv_l0_repair": 1309071616,
    "decompress:wzp_decode": 576808704,
    "decompress:inv_l0": 1053336576,
}


def algorithmic_bytes(n, s, a, fused=True):
    """Bytes each timed stage must move at least (its inputs read once and its
    outputs written once); a = archive bytes. Level kernels of the dyadic
    schedule: level 0 dominates (7/8 of the samples). With `fused` the WZP
    encoder quantises the coefficients itself (reads and rewrites them)."""
    w = a  # WZP stream is nearly the whole archive
    return {
        "compress:fwd_l0": 2 * n * s,
        "compress:quantize": 2 * n * s + 2 * n + n // 8,
        "compress:wzp_encode": (2 * n * s + w) if fused else (2 * n + n // 8 + w),
        "compress:inv_l0_repair": 2 * n * s,
        "decompress:wzp_decode": w + n * s,
        "decompress:inv_l0": 2 * n * s,
    }


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- CPU arms
def _codec(kind):
    from oracle import oracle as O
    if kind == "reference":
        return O.RefCodec(O.AVX2)
    class Port:
        compress = staticmethod(O.compress)
        decompress = staticmethod(O.decompress)
    return Port()


def cpu_baseline(field, eb, ours=None):
    """Reference CPU codec (oracle/_ref, AVX2; the C port when it is not
    built) on the same workload: the whole field as one archive, one
    compress and one decompress, timed separately. The codec has no threads
    of its own, so one archive runs on one core. With `ours`, also whether
    its archive equals ours byte for byte."""
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    codec = _codec(kind)
    t0 = time.perf_counter()
    a = codec.compress(field, eb)
    t1 = time.perf_counter()
    codec.decompress(a, field.shape, field.dtype)
    t2 = time.perf_counter()
    out = {"value": round(field.nbytes / (t2 - t0) / 1e9, 4), "unit": "GB/s", "cores": 1, "kind": kind,
           "compress_gbs": round(field.nbytes / (t1 - t0) / 1e9, 4),
           "decompress_gbs": round(field.nbytes / (t2 - t1) / 1e9, 4),
           "sample": f"the whole {'x'.join(str(d) for d in field.shape[::-1])} field as one archive, one "
                     f"compress + decompress, reference CPU codec "
                     f"{'AVX2 backend' if kind == 'reference' else '(C port)'}, 1 thread ({t2 - t0:.1f} s)"}
    if ours is not None and kind == "reference":
        out["archive_identical_to_ours"] = len(a) == ours.numel() and a == ours.cpu().numpy().tobytes()
    return out


def gpu_baseline(field, eb, ours, steps):
    """The reference's own CUDA library (oracle/_ref/libwaltz_refgpu.so, its
    src/waltz.cu and src/lossless/wzp.cu compiled for sm_100a) on the same
    field, bound and GPU: device-resident input, one compress and one
    decompress per step, CUDA events around each call, median over `steps`
    after two warm-up steps. Its archive is compared with ours byte for byte."""
    import torch
    from oracle import oracle as O
    if not O.refgpu_available():
        return {"unavailable": "reference CUDA library not built (make -C oracle refgpu)"}
    lib = O.refgpu_lib()
    shape, width = tuple(field.shape), field.element_size()
    src = field.clone()  # the reference takes a mutable input pointer
    arch = torch.empty(lib.refgpu_capacity(field.numel(), width), dtype=torch.uint8, device=field.device)
    out = torch.empty_like(field)
    stream = torch.cuda.current_stream().cuda_stream
    tc, td, size = [], [], 0
    for it in range(2 + steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        size = O.refgpu_compress(src.data_ptr(), width, shape, eb, arch.data_ptr(), stream)
        e[1].record()
        O.refgpu_decompress(arch.data_ptr(), width, shape, out.data_ptr(), stream)
        e[2].record()
        torch.cuda.synchronize()
        if it >= 2:
            tc.append(e[0].elapsed_time(e[1]))
            td.append(e[1].elapsed_time(e[2]))
    nbytes = field.numel() * width
    t_c, t_d = statistics.median(tc), statistics.median(td)
    identical = size == ours.numel() and bool(torch.equal(arch[:size], ours))
    worst = float((out.double() - field.double()).abs().max())
    del src, arch, out
    return {"value": round(nbytes / ((t_c + t_d) / 1e3) / 1e9, 3), "unit": "GB/s",
            "compress_gbs": round(nbytes / (t_c / 1e3) / 1e9, 3),
            "decompress_gbs": round(nbytes / (t_d / 1e3) / 1e9, 3),
            "ms_per_step": round(t_c + t_d, 4), "archive_bytes": size, "archive_identical_to_ours": identical,
            "max_abs_error": worst, "kind": "reference CUDA library, same GPU",
            "sample": f"same field and bound, {steps} steps after 2 warm-up, device-resident"}


def cpu_batch_baseline(chunks, bounds, budget_s=10.0):
    """Reference CPU codec (oracle/_ref, AVX2) over the chunk list with one
    workspace per thread (up to 8 threads), compress + decompress per chunk,
    until the list or about `budget_s` seconds are done."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    threads = max(1, min(8, os.cpu_count() or 1))
    local = __import__("threading").local()
    t0 = time.perf_counter()

    def work(i):
        if time.perf_counter() - t0 > budget_s:
            return 0
        if not hasattr(local, "codec"):
            local.codec = _codec(kind)
        a = local.codec.compress(chunks[i], bounds[i])
        local.codec.decompress(a, chunks[i].shape, chunks[i].dtype)
        return chunks[i].nbytes

    with ThreadPoolExecutor(threads) as pool:
        sizes = list(pool.map(work, range(len(chunks))))
    secs = time.perf_counter() - t0
    done = sum(sizes)
    return {"value": round(done / secs / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": kind,
            "sample": f"{sum(1 for x in sizes if x)} of {len(chunks)} chunks, compress + decompress each, reference "
                      f"CPU codec AVX2 backend, one workspace per thread ({secs:.1f} s)"}


def reference_arm(args):
    """The reference's CPU implementation of the path on this arm's workload:
    each step compresses the f32 512^3 field into one archive and decodes it
    again (oracle/_ref, AVX2 backend). The reference CPU codec has no threads
    of its own, so one archive uses one core whatever the host offers. Beside
    the line, `parallel_blocks` gives the codec's throughput when the same
    field is cut into independent blocks, one per host thread (another
    configuration: 8 or 64 archives instead of one)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    from waltz_b200.synthetic import power_law_field
    kind = "reference" if O.ref_available() else "port"
    shape = tuple(args.shape)
    field = power_law_field(shape, SEED)
    eb = REL * (float(field.max()) - float(field.min()))
    codec = _codec(kind)
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        a = codec.compress(field, eb)
        codec.decompress(a, field.shape, field.dtype)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    step = statistics.median(times)
    value = field.nbytes / step / 1e9
    # context: the same field as independent blocks, one per host thread
    threads = max(1, len(os.sched_getaffinity(0)))
    split = 2 if threads <= 8 else 4
    side = [d // split for d in field.shape]
    blocks = [np.ascontiguousarray(field[z * side[0]:(z + 1) * side[0], y * side[1]:(y + 1) * side[1],
                                         x * side[2]:(x + 1) * side[2]])
              for z in range(split) for y in range(split) for x in range(split)]
    cores = min(threads, len(blocks))
    local = threading.local()

    def work(i):
        if not hasattr(local, "codec"):
            local.codec = _codec(kind)
        b = blocks[i]
        local.codec.decompress(local.codec.compress(b, eb), b.shape, b.dtype)
        return b.nbytes

    with ThreadPoolExecutor(cores) as pool:
        t0 = time.perf_counter()
        done = sum(pool.map(work, range(len(blocks))))
        par = done / (time.perf_counter() - t0) / 1e9
    backend = "AVX2 backend" if kind == "reference" else "C port"
    dims = "x".join(str(d) for d in shape[::-1])
    sample = (f"f32 {dims} field as one archive, one compress + decompress per step, reference CPU codec "
              f"({backend}), 1 thread (the codec has none of its own)")
    return {"metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(step * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"f32 {'x'.join(str(d) for d in shape)} (z,y,x) k^-11/3 GRF seed 1, REL 1e-3, "
                                   "one archive, step = compress + decompress",
                       "parallelism": "1 host thread"},
            "impl": "reference",
            "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": 1, "kind": kind, "sample": sample},
            "parallel_blocks": {"value": round(par, 4), "unit": "GB/s", "cores": cores,
                                "sample": f"the same field as {len(blocks)} independent {side[0]}^3 archives, "
                                          f"compress + decompress each, {cores} threads, one pass"},
            "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gpu-baseline", action="store_true",
                    help="skip the reference CUDA library timed on the same GPU")
    ap.add_argument("--no-tc-form", action="store_true", help="skip the plain vs tensor-core form comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched vs per-chunk comparison")
    ap.add_argument("--tc-shape", type=int, nargs=3, default=[64, 1024, 1024], metavar=("NZ", "NY", "NX"),
                    help="field of the tensor-core comparison (z y x); smaller shapes serve profiler captures")
    ap.add_argument("--shape", type=int, nargs=3, default=list(SHAPE), metavar=("NZ", "NY", "NX"),
                    help="field shape (z y x); smaller shapes serve profiler captures")
    ap.add_argument("--batch-only", action="store_true",
                    help="run only the batched form on the uneven-chunk workload (profiler captures)")
    ap.add_argument("--tc-only", action="store_true",
                    help="run only the plain vs tensor-core form comparison at --tc-shape (profiler captures)")
    ap.add_argument("--batch-config", default=None, metavar="MODE:WIDTH[:STAGE[:ZMARCH]]",
                    help="batch execution form instead of the tuning table's (0 = stage-batched, 1 = field chains, "
                         "2 = work queues; STAGE: whole-stage plane kernels 1 or 0)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(reference_arm(args)))
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    if args.tc_only:
        import torch
        from waltz_b200 import _lib
        torch.cuda.set_device(local_rank)
        print(json.dumps(tc_form_comparison(torch.device("cuda", local_rank), _lib.lib(), args.steps,
                                            tuple(args.tc_shape), ref_gpu=False)))
        return
    if args.batch_only:
        import torch
        from waltz_b200 import _lib
        torch.cuda.set_device(local_rank)
        print(json.dumps(batch_only(torch.device("cuda", local_rank), _lib.lib(), args)))
        return
    try:
        result = gpu_arm(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(result))
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
