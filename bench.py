#!/usr/bin/env python
"""bench.py -- decoded MPix/s of the baseline-JPEG decode path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cudajpeg|reference]
                    [--workload mixed_batch|single_4096|single_1024|precision_8192]

Default workload (the batching configuration): one batch of 1024 seeded
synthetic baseline JPEGs, W and H log-uniform in [64, 2048], 4:2:0 / 4:2:2 /
4:4:4 / grey with p = .6/.2/.1/.1, quality U[50, 95], 30% with restart
intervals of 16-64 MCUs (about 320 MPix, 58 MB of JPEG).  One step = one
decode of the whole batch: one CUDA-graph launch of the persistent
cooperative decode kernel and the pixel kernel (cjBatchRun), under the
tuning the autotuner (cjBatchAutotune) picks in the untimed warm-up.
The single_* workloads time the plain per-image path (openJPG) instead;
precision_8192 is the iDCT precision A/B (run_precision).

* ``value``   device-resident throughput: the compressed bytes are already in
  HBM when the timed region starts; each step is timed with CUDA events on
  the decoder's stream.  The batch's working set (inputs, coefficients,
  outputs: ~1.6 GB) is far larger than L2; for the single-image workloads L2
  is flushed (256 MiB write) before every step, outside the events.  Max
  over ranks.
* ``e2e``     the same metric through the public C API: per step the host
  parse, the host->device copy of the files from pinned memory, the decode,
  and the device->host copy of every decoded image into pinned memory.
* ``roofline`` the dominant kernel (k_decode_batch): the path's algorithmic
  bytes (compressed scans read + decoded pixels written) / its duration
  (in-kernel %globaltimer phase stamps), against the measured HBM copy
  bandwidth in MEASURED_PEAKS.json (else the fallback figure, said so);
  ``kernel_min_bytes`` adds the kernel's own intermediates (destuffed copy
  written and read twice, int16 coefficient blocks written);
  ``roofline_pixel`` the same for k_pixel_batch (its algorithmic bytes are
  the pixels it writes; ``kernel_min_bytes`` adds the blocks it reads).
* ``plain_path`` (batch workload) the per-image path over the same images.
* ``serving`` open-loop Poisson request streams through the continuous-
  batching server (cudajpeg_b200.serve): p50/p99/p99.9 latency, MPix/s.
* ``cpu_baseline`` the reference's own CPUonly decoder (compiled from its
  sources into oracle/_ref) on the host cores, on a bounded sample.

``--impl reference`` times only that CPU decoder (all host threads) on the
same workload and prints the same metric with "impl": "reference".
Multi-GPU (torchrun): every rank decodes its own replica of the workload (no
collective on the data path; images are independent) -> "scaling": "weak".
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "decoded MPix/s"
FLUSH_BYTES = 256 << 20

# Minimum bytes of each kernel of the single-image path, per launch, as a
# function of the image: B = entropy-coded bytes, Bd = destuffed bytes,
# n = 8x8 blocks, P = output bytes.  k_decode_batch reads the compressed
# scan, writes the destuffed copy, reads it twice (speculative sync and
# write-out) and writes the int16 blocks; k_pixel reads the blocks and
# writes the image.
KERNEL_BYTES = {
    "k_decode_batch": lambda g: g["B"] + 3 * g["Bd"] + 128 * g["n"],
    "k_pixel": lambda g: 128 * g["n"] + g["P"],
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cudajpeg", choices=["cudajpeg", "reference"])
    ap.add_argument("--workload", default="mixed_batch",
                    choices=["mixed_batch", "single_4096", "single_1024", "precision_8192"])
    ap.add_argument("--precision-size", type=int, default=8192,
                    help="image side of the precision workload (8192 as specified)")
    ap.add_argument("--batch-size", type=int, default=1024)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the single-image and precision configurations in the default run")
    ap.add_argument("--split", action="store_true",
                    help="under torchrun: partition one batch across ranks (strong scaling) "
                         "instead of one batch per rank (weak scaling)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default batch tuning")
    ap.add_argument("--idct", default="tc", choices=["int", "tc"],
                    help="pixel-stage iDCT of the batch: tensor cores (the metric's batched+TC-iDCT form, "
                         "samples within +-1 of the reference) or the reference's integer iDCT (bit-exact); "
                         "the other form is reported beside it")
    ap.add_argument("--kernels-only", action="store_true",
                    help="time the batch run only (no end-to-end, plain path, serving or other configurations): "
                         "the short command the profiles are captured with")
    ap.add_argument("--tuning", default="",
                    help="fixed batch tuning SUB_BITS,CTAS_PER_SM,TILE_CAP instead of the autotuner")
    ap.add_argument("--host-parse", action="store_true",
                    help="parse the batch's marker segments on the host instead of the GPU (cjBatchSetParse)")
    ap.add_argument("--serve-seconds", type=float, default=1.5,
                    help="seconds of arrivals per rate for the serving measurement (0: skip)")
    return ap.parse_args()


class Workload:
    """The files of one step, their pixel count and the JSON `config`.
    Under torchrun the mixed batch is per rank: its own seed (weak scaling)
    or its share of one batch (strong scaling, --split)."""

    def __init__(self, name: str, batch_size: int, rank: int = 0, world: int = 1, split: bool = False):
        from cudajpeg_b200 import replicas as R
        from cudajpeg_b200 import workloads as W
        self.name = name
        if name == "mixed_batch":
            workers = max(1, min(32, (os.cpu_count() or 1) // world))
            seed = 4 if split else R.rank_seed(4, rank)
            samples = W.mixed_batch(n=batch_size, seed=seed, workers=workers)
            if split and world > 1:
                share = R.partition([s.pixels for s in samples], world)[rank]
                samples = [samples[i] for i in share]
            self.config = {"workload": f"mixed_batch_{batch_size}", "images": batch_size,
                           "sides": "log-uniform [64, 2048], multiples of 8",
                           "subsampling": "4:2:0/4:2:2/4:4:4/grey p=.6/.2/.1/.1",
                           "quality": "U[50, 95]",
                           "restart": "30% with 16-64 MCU intervals"}
        else:
            samples = [W.single_4096() if name == "single_4096" else W.single_1024()]
            s = samples[0]
            self.config = {"workload": f"{name}_{s.mode}_q{s.quality}", "images": 1,
                           "width": s.width, "height": s.height, "subsampling": s.mode,
                           "quality": s.quality, "restart": s.restart}
        self.samples = samples
        self.files = [s.data for s in samples]
        self.pixels = sum(s.pixels for s in samples)
        self.out_bytes = sum(s.pixels * (1 if s.mode == "gray" else 3) for s in samples)
        self.file_bytes = sum(len(f) for f in self.files)
        self.config.update({"MPix": round(self.pixels / 1e6, 3), "file_MB": round(self.file_bytes / 1e6, 3),
                            "data": "synthetic, seeded (cudajpeg_b200/workloads.py); Pillow/libjpeg "
                                    "encoder, Annex K Huffman tables"})


# ---------------------------------------------------------------- CPU baseline

def ref_cpu_time(files, threads: int, budget_s: float):
    """Time the reference CPUonly decoder (oracle/_ref) -- or, if that build is
    absent, the oracle port -- decoding `files` from /dev/shm, one image per
    thread at a time on `threads` threads, for about `budget_s` seconds.
    Returns (kind, seconds, decoded pixels, failed decodes)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    d = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    tmp = tempfile.mkdtemp(dir=d)
    paths = []
    for k, data in enumerate(files):
        p = os.path.join(tmp, f"{k}.jpg")
        with open(p, "wb") as f:
            f.write(data)
        paths.append(p)
    try:
        if O.ref_available():
            secs, px, fails = O.ref_cpu_bench(paths, 1, threads)  # one pass calibrates
            iters = max(1, int(budget_s / max(secs, 1e-3)))
            if iters > 1:
                secs, px, fails = O.ref_cpu_bench(paths, iters, threads)
            else:
                iters = 1
            return "reference", secs, px, fails
        from concurrent.futures import ThreadPoolExecutor

        def one(data):
            r = O.decode(data)
            return (r.width * r.height, 0) if r.error == 0 else (0, 1)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            res = list(ex.map(one, files))
        secs = time.perf_counter() - t0
        return "port", secs, sum(r[0] for r in res), sum(r[1] for r in res)
    finally:
        for p in paths:
            os.unlink(p)
        os.rmdir(tmp)


REF_HOW = ("the reference's CPUonly openJPG (CPUonly/src/main.c:10); files with restart markers, "
           "which CPUonly rejects (CPUonly/src/decodeScanCPU.c:41-43), through the reference's GPU-tree "
           "host decoder (src/decodeScanCPU.cu:98-152) + CPUonly iDCT_row/iDCT_col, upsampling and colour")


def cpu_baseline(wl: Workload, threads: int, budget_s: float) -> dict:
    kind, secs, px, fails = ref_cpu_time(wl.files, threads, budget_s)
    who = REF_HOW if kind == "reference" else "oracle port of the reference path"
    note = f"; {fails} decodes failed and their pixels are not counted" if fails else ""
    return {"value": round(px / secs / 1e6, 3), "unit": "MPix/s", "cores": threads, "kind": kind,
            "sample": f"{px / 1e6:.1f} MPix decoded in {secs:.1f} s from /dev/shm, "
                      f"{wl.config['workload']} files ({who}; one image per thread){note}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = Workload(args.workload, args.batch_size)
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        O.build()
    times, pix, fails = [], 0, 0
    for k in range(args.warmup + args.steps):
        # each step decodes the workload's files once, spread over all threads
        kind, secs, px, f = ref_cpu_time(wl.files, threads, 0.0)
        if k >= args.warmup:
            times.append(secs)
            pix += px
            fails = f
    total = sum(times)
    value = pix / total / 1e6
    note = f"; {fails} of {len(wl.files)} files failed and their pixels are not counted" if fails else ""
    line = {"metric": METRIC, "value": round(value, 3), "unit": "MPix/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic",
            "config": wl.config, "impl": "reference",
            "cpu_baseline": {"value": round(value, 3), "unit": "MPix/s", "cores": threads,
                             "kind": kind,
                             "sample": f"each step decodes the {len(wl.files)} workload files once "
                                       f"on {threads} threads from /dev/shm: {REF_HOW}{note}"},
            "e2e": {"value": round(value, 3), "unit": "MPix/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[1].isdigit():
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [int(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- GPU arm

def read_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def traffic_key(workload: str, batch_size: int) -> str:
    """Name of the committed ncu summary that holds DRAM bytes per launch for
    this run: the summaries are captured on the default 1024-image batch, so
    other batch sizes look for a summary of their own (and report null)."""
    return workload if batch_size == 1024 else f"{workload}_{batch_size}"


def read_traffic(kernel: str, workload: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def plain_path_value(cj, files) -> dict:
    """The plain per-image path over the same files: device-resident re-decode
    of each image (cjReaderRedecodeDevice), device time summed."""
    import torch
    r = cj.Reader()
    ext = None
    total_ms, px = 0.0, 0
    for data in files:
        if r.open_bytes(data, check=False):
            continue
        if ext is None:  # the reader's stream exists after its first decode
            ext = torch.cuda.ExternalStream(r.stream())
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(ext)
        r.redecode_device()
        e.record(ext)
        e.synchronize()
        total_ms += s.elapsed_time(e)
        inf = r.info()
        px += inf["width"] * inf["height"]
    r.close()
    return {"value": round(px / total_ms / 1e3, 2), "unit": "MPix/s",
            "how": "openJPG per image, then cjReaderRedecodeDevice timed with CUDA events "
                   "per image, summed over the same files"}


def serving_value(wl, seconds: float) -> dict:
    """Open-loop Poisson request streams of the workload's files (one JPEG
    per request) through the continuous-batching server at 2k, 8k and 32k
    requests/s; latency = scheduled arrival -> the request's batch finished
    on the GPU, outputs left on the device."""
    import numpy as np

    from cudajpeg_b200 import serve as sv
    px = np.array([s.pixels for s in wl.samples], np.float64)
    out = {"how": f"cjServerReplay, {seconds:g} s of Poisson arrivals per rate over the "
                  f"{len(wl.files)} workload files (cycled), 3 engines, 8 GiB budget, server "
                  "default tuning (512-bit subsequences)",
           "rates": []}
    with sv.Server(engines=3, hbm_budget_bytes=8 << 30, max_batch=256) as s:
        # warm-up: bursts of the largest files grow every engine's buffers to
        # steady-state size before any measured stream
        sizes = np.array([len(f) for f in wl.files])
        for idx in (np.argsort(-px)[:256], np.argsort(-sizes)[:256]):
            big = [wl.files[i] for i in idx]
            for _ in range(3):
                s.replay(big, np.zeros(3 * len(big)))
        s.replay(wl.files, sv.poisson_arrivals(8000.0, 4000, seed=99))
        for rate in (2000.0, 8000.0, 32000.0):
            n = int(rate * seconds)
            run = s.replay(wl.files, sv.poisson_arrivals(rate, n, seed=7))
            summ = sv.summarize(run, px, rate)
            out["rates"].append({k: (round(v, 3) if isinstance(v, float) else v) for k, v in summ.items()})
        out["server_stats"] = s.stats()
    return out


def batch_form_value(args, src, offsets, sizes, tune, wl, dist, idct_name: str) -> dict:
    """Device-resident MPix/s of the batch decoded with the other pixel-stage
    iDCT (cjBatchSetOutput(RGB, idct)) under the same tuning, and its pixel
    kernel's time."""
    import torch

    import cudajpeg_b200 as cj
    from cudajpeg_b200 import replicas as R
    idct = cj.IDCT_TC if idct_name == "tc" else cj.IDCT_INT
    with cj.Batch() as b:
        b.set_tuning(tune["sub_bits"], tune["decode_ctas_per_sm"], tune["pixel_tile_cap"])
        b.set_output(cj.OUTPUT_RGB, idct)
        b.stage(src.data_ptr(), offsets, sizes)
        ext = torch.cuda.ExternalStream(b.stream())
        for _ in range(args.warmup):
            b.run()
        if any(b.wait()):
            raise RuntimeError(f"batch decode errors ({idct_name} iDCT)")
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        pix = []
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            starts[k].record(ext)
            b.run()
            ends[k].record(ext)
            b.wait()
            pix.append(b.phase_ms()["pixel"])
        torch.cuda.synchronize()
        total = R.max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(starts, ends)), dist, "cuda")
        job_pixels = R.sum_over_ranks(wl.pixels, dist, "cuda")
    how = {"tc": "k_pixel_batch with the tcgen05 FP16 hi/lo iDCT (FP32 accumulation in tensor memory)",
           "int": "k_pixel_batch with the reference's integer iDCT (bit-exact pixels)"}[idct_name]
    return {"value": round(job_pixels * args.steps / (total / 1e3) / 1e6, 2), "unit": "MPix/s",
            "ms_per_step": round(total / args.steps, 4), "pixel_kernel_ms": round(statistics.mean(pix), 4),
            "how": how + ", same batch and tuning, CUDA events on the decoder's stream"}


def run_batch(args, wl, world, rank, local, dist):
    import numpy as np
    import torch

    import cudajpeg_b200 as cj
    from cudajpeg_b200 import replicas as R

    blob, offsets, sizes = cj.Batch.pack(wl.files)
    src = torch.empty(len(blob), dtype=torch.uint8, pin_memory=True)
    src.numpy()[:] = blob
    idct = cj.IDCT_TC if args.idct == "tc" else cj.IDCT_INT
    b = cj.Batch()
    b.set_parse(not args.host_parse)
    b.set_output(cj.OUTPUT_RGB, idct)
    b.stage(src.data_ptr(), offsets, sizes)
    b.run()
    b.fetch()
    errs = b.wait()
    if any(errs):
        raise RuntimeError(f"batch decode errors: {sum(1 for e in errs if e)}")
    # untimed: the autotuner picks subsequence size, decode-kernel occupancy
    # and pixel tile width for this batch (cjBatchAutotune)
    if args.tuning:
        b.set_tuning(*[int(x) for x in args.tuning.split(",")])
        b.stage(src.data_ptr(), offsets, sizes)
        tune = b.tuning()
    elif args.no_autotune:
        tune = b.tuning()
    else:
        tune = b.autotune(src.data_ptr(), offsets, sizes, reps=3)
    b.run()
    if any(b.wait()):
        raise RuntimeError("batch decode errors under the tuned configuration")
    ext = torch.cuda.ExternalStream(b.stream())
    for _ in range(args.warmup):
        b.run()
    b.wait()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    phases: dict = {}
    launches0 = b.stats()["launches"]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            starts[k].record(ext)
            b.run()
            ends[k].record(ext)
            if any(b.wait()):
                raise RuntimeError("batch run reported image errors")
            for name, ms in b.phase_ms().items():
                phases.setdefault(name, []).append(ms)
        torch.cuda.synchronize()
    st_run = b.stats()
    launches = st_run["launches"] - launches0
    if dist:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    # whole job: pixels of all ranks / the slowest rank's device time
    total_ms = R.max_over_ranks(sum(step_ms), dist, "cuda")
    job_pixels = R.sum_over_ranks(wl.pixels, dist, "cuda")
    job_file_bytes = R.sum_over_ranks(wl.file_bytes, dist, "cuda")
    value = job_pixels * args.steps / (total_ms / 1e3) / 1e6
    if args.kernels_only:
        b.close()
        return {"metric": METRIC, "value": round(value, 2), "unit": "MPix/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32",
                "data": "synthetic", "config": dict(wl.config, idct=args.idct, kernels_only=True,
                                                   tuning=tune),
                "phase_ms": {k: round(statistics.mean(v), 4) for k, v in phases.items()},
                "gpu_launches": int(launches), "clocks": clocks.summary()}

    # end to end through the public C API: every step parses the files on the
    # host, copies them from pinned memory to the device, decodes, and copies
    # every decoded image back to pinned memory.  Two batch decoders alternate
    # (each with its own stream), so one step's device->host copy overlaps the
    # next step's host->device copy, marker parse (on the GPU) and kernels.
    b2 = cj.Batch()
    b2.set_parse(not args.host_parse)
    b2.set_tuning(tune["sub_bits"], tune["decode_ctas_per_sm"], tune["pixel_tile_cap"])
    b2.set_output(cj.OUTPUT_RGB, idct)
    pair = [b, b2]
    e2e_lat = []
    for x in pair:  # one sequential step each: latency of a lone step, and buffers warm
        t0 = time.perf_counter()
        x.stage(src.data_ptr(), offsets, sizes)
        x.run()
        x.fetch()
        if any(x.wait()):
            raise RuntimeError("batch decode errors")
        e2e_lat.append(1e3 * (time.perf_counter() - t0))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        x = pair[k & 1]
        x.stage(src.data_ptr(), offsets, sizes)
        x.run()
        x.fetch()
        if k and any(pair[(k - 1) & 1].wait()):
            raise RuntimeError("batch decode errors")
    if any(pair[(args.steps - 1) & 1].wait()):
        raise RuntimeError("batch decode errors")
    e2e_total = R.max_over_ranks(1e3 * (time.perf_counter() - t0), dist, "cuda")
    e2e_value = job_pixels * args.steps / (e2e_total / 1e3) / 1e6
    st = b.stats()
    b.close()
    b2.close()

    peaks = read_peaks()
    mean_ms = total_ms / args.steps
    pm = {k: round(statistics.mean(v), 4) for k, v in phases.items()}
    # per-kernel rooflines from the in-kernel phase stamps (CUDA-event total
    # split by %globaltimer stamps at each phase start and the pixel kernel's end)
    decode_ms = sum(pm[k] for k in cj.BATCH_PHASES[:9])
    pixel_ms = pm["pixel"]
    coef_bytes = st_run["blocks"] * 128
    # The path's algorithmic bytes are the compressed scans read
    # plus the decoded pixels written; intermediates are not counted.  The
    # dominant kernel is k_decode_batch, so the roofline is those bytes over
    # its time; the same bytes over the whole step, and each kernel's own
    # minimum with its intermediates (destuffed copy written and read twice,
    # int16 blocks written / read), are reported beside it.
    alg_path = st_run["input_bytes"] + st_run["output_bytes"]
    min_decode = st_run["input_bytes"] + 3 * st_run["scan_bytes"] + coef_bytes
    min_pixel = coef_bytes + st_run["output_bytes"]
    ach_decode = alg_path / (decode_ms / 1e3) / 1e9
    ach_step = alg_path / (mean_ms / 1e3) / 1e9
    tkey = traffic_key(args.workload, args.batch_size)
    # the pixel kernel's share of the path's algorithmic bytes: the pixels it
    # writes (its int16 block reads are an intermediate, kernel_min_bytes)
    ach_pixel = st_run["output_bytes"] / (pixel_ms / 1e3) / 1e9
    ach_pixel_min = min_pixel / (pixel_ms / 1e3) / 1e9
    tr_decode = read_traffic("k_decode_batch", tkey)
    tr_pixel = read_traffic("k_pixel_batch", tkey + ("_tc" if args.idct == "tc" else ""))
    tr_step = tr_decode + tr_pixel if tr_decode and tr_pixel else None
    line = {"metric": METRIC, "value": round(value, 2), "unit": "MPix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(mean_ms, 4),
            "higher_is_better": True, "scaling": "strong" if args.split else "weak",
            "vs_baseline": None,
            "dtype": ("u8/int16 entropy; iDCT fp16 hi/lo x fp32 accumulate (tensor cores)" if args.idct == "tc"
                      else "u8/int16/int32"),
            "data": "synthetic",
            "config": dict(wl.config, idct=args.idct, marker_parse="host" if args.host_parse else "gpu",
                           parallelism=(f"split{world}: one batch partitioned by pixels" if args.split
                                        else f"shards{world}: one batch per rank, seed 4 + rank"),
                           l2="working set ~1.6 GB per step, larger than L2 (126 MB)",
                           job_MPix=round(job_pixels / 1e6, 3),
                           compressed_MB_per_s=round(job_file_bytes * args.steps
                                                     / (total_ms / 1e3) / 1e6, 1),
                           passes=st["passes"], grid_ctas=st["grid"], warp_items=st["warp_items"],
                           pixel_ctas=st["pixel_grid"],
                           tuning={k: tune[k] for k in ("sub_bits", "decode_ctas_per_sm", "pixel_tile_cap",
                                                        "sub_bits_class") if k in tune},
                           autotune=({"best_ms": tune["best_ms"], "trials_ms": tune["trials_ms"],
                                      "order": "sub_bits {512,1024,2048,4096} x ctas {3,4,5}, then per "
                                               "sampling class (4:2:0, 4:2:2, 4:4:4, grey, other; classes "
                                               "with >= 1/16 of the scan bytes) sub_bits {1024..16384}, "
                                               "then tile cap {8,4,2}"}
                                     if "best_ms" in tune else None)),
            "e2e": {"value": round(e2e_value, 2), "unit": "MPix/s",
                    "h2d_bytes_per_step": int(st["input_bytes"]),
                    "d2h_bytes_per_step": int(st["output_bytes"]),
                    "ms_per_step": round(e2e_total / args.steps, 3),
                    "lone_step_ms": round(min(e2e_lat), 3),
                    "how": "two cjBatch decoders alternate: step k's D2H overlaps step k+1's marker parse (GPU), "
                           "H2D and kernels; every step's copies are inside the timed region"},
            "roofline": {"bound": "hbm", "kernel": "k_decode_batch", "achieved": round(ach_decode, 1),
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(ach_decode / peaks["hbm_gbs"], 4),
                         "traffic": tr_decode,
                         "algorithmic_bytes": int(alg_path), "kernel_ms": round(decode_ms, 4),
                         "kernel_min_bytes": int(min_decode),
                         "bytes": "compressed scans read + decoded pixels written (per batch); "
                                  "kernel_min_bytes adds the kernel's own intermediates",
                         "peak_source": peaks["source"]},
            "roofline_step": {"bound": "hbm", "kernels": "k_decode_batch + k_pixel_batch",
                              "achieved": round(ach_step, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                              "frac": round(ach_step / peaks["hbm_gbs"], 4), "algorithmic_bytes": int(alg_path),
                              "traffic": tr_step,
                              "traffic_over_algorithmic": (round(tr_step / alg_path, 3) if tr_step else None),
                              "ms": round(mean_ms, 4)},
            "roofline_pixel": {"bound": "hbm", "kernel": "k_pixel_batch", "achieved": round(ach_pixel, 1),
                               "peak": peaks["hbm_gbs"], "unit": "GB/s",
                               "frac": round(ach_pixel / peaks["hbm_gbs"], 4),
                               "traffic": tr_pixel,
                               "algorithmic_bytes": int(st_run["output_bytes"]),
                               "kernel_min_bytes": int(min_pixel), "kernel_ms": round(pixel_ms, 4),
                               "achieved_kernel_min": round(ach_pixel_min, 1),
                               "bytes": "decoded pixels written (algorithmic); kernel_min_bytes adds the "
                                        "int16 blocks it reads",
                               "peak_source": peaks["source"]},
            "phase_ms": pm, "gpu_launches": int(launches), "clocks": clocks.summary()}
    # the same batch with the tensor-core iDCT in the pixel kernel (the
    # metric's batched + TC-iDCT form; output within +-1 per sample of the
    # integer iDCT's), timed the same way
    other = "int" if args.idct == "tc" else "tc"
    alt = batch_form_value(args, src, offsets, sizes, tune, wl, dist, other)
    line[f"batched_{other}"] = alt
    if rank == 0 and world == 1:
        line["plain_path"] = plain_path_value(cj, wl.files)
        line["plain_path"]["batched_over_plain"] = round(value / line["plain_path"]["value"], 2)
        line["plain_path"][f"batched_{other}_over_plain"] = round(alt["value"] / line["plain_path"]["value"], 2)
        if args.serve_seconds > 0:
            line["serving"] = serving_value(wl, args.serve_seconds)
    return line


def run_single(args, wl, world, rank, local, dist):
    """The plain per-image path (openJPG / cjReaderRedecodeDevice) on one
    image: device time per decode with L2 flushed before each, and the end
    to end call (host parse, copies, kernels) per decode."""
    import numpy as np
    import torch

    import cudajpeg_b200 as cj
    from cudajpeg_b200 import replicas as R

    sample = wl.samples[0]
    n = len(sample.data)
    src = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    src.numpy()[:] = np.frombuffer(sample.data, np.uint8)
    reader = cj.Reader()
    reader.open_bytes((src.data_ptr(), n))
    info = reader.info()
    ext = torch.cuda.ExternalStream(reader.stream())
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    nblocks = info["mcux"] * info["mcuy"] * info["bpm"]
    geom = {"B": info["scan_bytes"], "Bd": info["destuffed"], "n": nblocks, "P": wl.out_bytes}
    for _ in range(args.warmup):
        reader.redecode_device()
    reader.open_bytes((src.data_ptr(), n))
    torch.cuda.synchronize()
    if reader.sync():
        raise RuntimeError("warm-up decode reported an error")
    reader.set_profile(True)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kern_ms: dict = {}
    launches0 = reader.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(ext):
                flush.zero_()
                starts[k].record(ext)
            reader.redecode_device()
            ends[k].record(ext)
            ext.synchronize()
            for name, ms in reader.kernel_times():
                kern_ms.setdefault(name, []).append(ms)
        torch.cuda.synchronize()
    launches = reader.launch_count() - launches0
    if dist:
        dist.barrier()
    if reader.sync():
        raise RuntimeError("device decode reported an error")
    reader.set_profile(False)
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = R.max_over_ranks(sum(step_ms), dist, "cuda")
    job_pixels = R.sum_over_ranks(wl.pixels, dist, "cuda")  # each rank decodes its own copy
    value = job_pixels * args.steps / (total_ms / 1e3) / 1e6
    e2e_ms = []
    if dist:
        dist.barrier()
    for _ in range(args.steps):
        with torch.cuda.stream(ext):
            flush.zero_()
        ext.synchronize()
        t0 = time.perf_counter()
        reader.open_bytes((src.data_ptr(), n))
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_total = R.max_over_ranks(sum(e2e_ms), dist, "cuda")
    e2e_value = job_pixels * args.steps / (e2e_total / 1e3) / 1e6
    means = {k: statistics.mean(v) for k, v in kern_ms.items()}
    dom = max(means, key=means.get)
    peaks = read_peaks()
    # The path's algorithmic bytes (compressed scan read + pixels written)
    # over the dominant kernel's time; the kernel's own minimum bytes beside
    alg = geom["B"] + geom["P"]
    achieved = alg / (means[dom] / 1e3) / 1e9
    reader.close()
    return {"metric": METRIC, "value": round(value, 2), "unit": "MPix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32", "data": "synthetic",
            "config": dict(wl.config, parallelism=f"replicas{world}",
                           l2="flushed before each step (256 MiB write, outside the timing)",
                           compressed_MB_per_s=round(world * info["scan_bytes"] * args.steps
                                                     / (total_ms / 1e3) / 1e6, 1)),
            "latency_ms": {"device_p50": round(float(np.percentile(step_ms, 50)), 4),
                           "device_p99": round(float(np.percentile(step_ms, 99)), 4),
                           "e2e_p50": round(float(np.percentile(e2e_ms, 50)), 4),
                           "e2e_p99": round(float(np.percentile(e2e_ms, 99)), 4)},
            "e2e": {"value": round(e2e_value, 2), "unit": "MPix/s",
                    "h2d_bytes_per_step": info["scan_bytes"] + info["param_bytes"],
                    "d2h_bytes_per_step": wl.out_bytes + 32,
                    "ms_per_step": round(e2e_total / args.steps, 3),
                    "how": "openJPGMem per step from pinned host memory: host parse, H2D copy of the "
                           "scan and tables, kernels, D2H copy of the image, all inside the timed region"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4),
                         "traffic": read_traffic(dom, args.workload), "algorithmic_bytes": int(alg),
                         "kernel_min_bytes": int(KERNEL_BYTES[dom](geom)),
                         "kernel_ms": round(means[dom], 4), "peak_source": peaks["source"]},
            "kernel_ms": {k: round(v, 4) for k, v in means.items()},
            "gpu_launches": int(launches), "clocks": clocks.summary()}


def idct_basis_f64():
    """C[u, x] = c(u)/2 cos((2x+1) u pi / 16), c(0) = 1/sqrt(2): the 8-point
    inverse DCT of T.81 A.3.3, in float64."""
    import numpy as np
    u = np.arange(8)[:, None]
    x = np.arange(8)[None, :]
    cu = np.where(u == 0, 1 / np.sqrt(2), 1.0)
    return cu / 2 * np.cos((2 * x + 1) * u * np.pi / 16)


def precision_line(args, steps: int, warmup: int, size: int) -> dict:
    """Precision form: plane iDCT of size x size q95 images (4:4:4, 4:2:2,
    grey; 50/50 uniform noise and gradient) in the three arithmetic forms of
    cjIDCTPlane -- the bit-exact fixed-point iDCT, FP32 on CUDA cores, FP16
    hi+lo basis on tensor cores with FP32 accumulation -- timed with CUDA
    events (L2 flushed before each launch), with the raw FP32 outputs
    (cjIDCTBlocksRaw) compared on the GPU against a float64 iDCT of the same
    dequantised coefficients, and the pixels against the integer form."""
    import numpy as np
    import torch

    import cudajpeg_b200 as cj
    from cudajpeg_b200 import workloads as W
    samples = [W.precision_8192(m, size=size) for m in ("444", "422", "gray")]
    basis = torch.from_numpy(idct_basis_f64()).cuda()
    peaks = read_peaks()
    modes = {"int": cj.IDCT_INT, "f32": cj.IDCT_F32, "tc": cj.IDCT_TC}
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    ones = torch.ones(64, dtype=torch.int16, device="cuda")
    rows = []
    tot = {m: [0.0, 0] for m in modes}
    worst = {"f32": 0.0, "tc": 0.0}
    for smp in samples:
        with cj.Reader(host_coefficients=True) as r:
            r.open_bytes(smp.data)
            coefs = r.coefficients()  # dequantised int32 per component, reference layout
            for c in range(len(coefs)):
                g = r.plane_geometry(c)
                nblk = coefs[c].shape[0]
                planes, ms = {}, {}
                stream = torch.cuda.current_stream()
                for name, mode in modes.items():
                    out = torch.zeros((g["rows"], g["stride"]), dtype=torch.uint8, device="cuda")
                    for _ in range(warmup):
                        r.plane_launch(g, out.data_ptr(), mode, stream.cuda_stream)
                    ts = []
                    for _ in range(steps):
                        flush.zero_()  # coefficients (128 B/block) start outside L2
                        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        s0.record(stream)
                        r.plane_launch(g, out.data_ptr(), mode, stream.cuda_stream)
                        s1.record(stream)
                        s1.synchronize()
                        ts.append(s0.elapsed_time(s1))
                    ms[name] = float(np.median(ts))
                    planes[name] = out
                    tot[name][0] += ms[name]
                    tot[name][1] += nblk * 64
                ref = planes["int"].to(torch.int16)
                match = {}
                for name in ("f32", "tc"):
                    d = (planes[name].to(torch.int16) - ref).abs()
                    match[name] = {"exact": round(float((d == 0).double().mean()), 6),
                                   "within_1": round(float((d <= 1).double().mean()), 6),
                                   "max_abs": int(d.max())}
                # raw (pre-rounding) error against float64, in chunks on the GPU
                deq = coefs[c]
                if np.abs(deq).max() > 32767:
                    raise RuntimeError("dequantised coefficient outside int16")
                dev = torch.from_numpy(deq.astype(np.int16)).cuda()
                err = {}
                for name in ("f32", "tc"):
                    mx, sm = 0.0, 0.0
                    for k0 in range(0, nblk, 1 << 18):
                        blk = dev[k0:k0 + (1 << 18)].contiguous()
                        raw = cj.idct_blocks_raw_device(blk, ones, modes[name])
                        x = blk.double().view(-1, 8, 8)
                        want = (basis.t() @ x @ basis).reshape(-1, 64)   # out[y][x] = sum_vu C[v,y] C[u,x] F[v,u]
                        e = (raw.double() - want).abs()
                        mx = max(mx, float(e.max()))
                        sm += float(e.sum())
                    err[name] = {"max_abs_vs_f64": round(mx, 6), "mean_abs_vs_f64": round(sm / (nblk * 64), 8)}
                    worst[name] = max(worst[name], mx)
                mpix = {k: round(nblk * 64 / (v / 1e3) / 1e6, 1) for k, v in ms.items()}
                gbs = {k: round(nblk * 192 / (v / 1e3) / 1e9, 1) for k, v in ms.items()}
                rows.append({"image": f"{smp.mode}_{smp.width}x{smp.height}_q{smp.quality}", "component": c,
                             "blocks": nblk, "ms": {k: round(v, 4) for k, v in ms.items()},
                             "MPix_per_s": mpix, "GB_per_s": gbs, "match_vs_int": match, "raw_error": err})
    tc_mpix = tot["tc"][1] / (tot["tc"][0] / 1e3) / 1e6
    tc_gbs = tot["tc"][1] * 3 / (tot["tc"][0] / 1e3) / 1e9   # 2 B coefficient in + 1 B sample out per pixel
    exact = {k: round(min(r_["match_vs_int"][k]["exact"] for r_ in rows), 6) for k in ("f32", "tc")}
    within = {k: round(min(r_["match_vs_int"][k]["within_1"] for r_ in rows), 6) for k in ("f32", "tc")}
    return {"metric": "plane iDCT MPix/s (tensor-core FP16 hi/lo, FP32 accumulate)", "value": round(tc_mpix, 1),
            "unit": "MPix/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": round(tot["tc"][0] / max(1, len(rows)), 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp16 hi/lo in, fp32 accumulate",
            "data": "synthetic",
            "config": {"workload": f"precision_{size}", "images": "444, 422, grey at q95",
                       "content": "50/50 uniform noise and gradient (cudajpeg_b200/workloads.py)",
                       "l2": "L2 flushed (256 MB write) before every timed launch"},
            "per_mode_MPix_per_s": {k: round(v[1] / (v[0] / 1e3) / 1e6, 1) for k, v in tot.items()},
            "max_abs_error_vs_f64": {k: round(v, 6) for k, v in worst.items()},
            "error_below_0_5": {k: v < 0.5 for k, v in worst.items()},
            "min_exact_fraction_vs_int": exact, "min_within_1_fraction_vs_int": within,
            "roofline": {"bound": "hbm", "kernel": "k_idct_tc", "achieved": round(tc_gbs, 1),
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(tc_gbs / peaks["hbm_gbs"], 4),
                         "traffic": read_traffic("k_idct_tc", f"precision_{size}"),
                         "peak_source": peaks["source"]},
            "rows": rows}


def run_precision(args):
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(precision_line(args, args.steps, args.warmup, args.precision_size)), flush=True)


def other_configs(args) -> dict:
    """The other benchmark configurations, measured in the default run at
    fewer steps: the plain per-image path on the 1024x768 and 4096x4096
    single images (MPix/s and p50/p99 latency), and the precision A/B of the
    plane iDCT forms on the 8192x8192 images."""
    out = {}
    for name in ("single_1024", "single_4096"):
        a = argparse.Namespace(**vars(args))
        a.steps, a.warmup, a.workload = 20, 3, name
        wl = Workload(name, 1)
        line = run_single(a, wl, 1, 0, 0, None)
        out[name] = {k: line[k] for k in ("value", "unit", "ms_per_step", "latency_ms", "e2e", "roofline",
                                          "kernel_ms", "gpu_launches", "clocks")}
        out[name]["config"] = line["config"]
    p = precision_line(args, 5, 3, args.precision_size)
    out[f"precision_{args.precision_size}"] = {k: p[k] for k in (
        "value", "unit", "per_mode_MPix_per_s", "max_abs_error_vs_f64", "error_below_0_5",
        "min_exact_fraction_vs_int", "min_within_1_fraction_vs_int", "roofline", "config")}
    return out


def run_gpu(args):
    import torch

    from cudajpeg_b200 import replicas as R
    rank, local, world = R.rank_env()
    # the workload is generated in a spawn-started pool before CUDA starts
    wl = Workload(args.workload, args.batch_size, rank, world, args.split)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    if args.workload == "mixed_batch":
        line = run_batch(args, wl, world, rank, local, dist)
    else:
        line = run_single(args, wl, world, rank, local, dist)
    if rank == 0 and world == 1 and args.workload == "mixed_batch" and not args.no_other_configs \
            and not args.kernels_only:
        line["other_configs"] = other_configs(args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.kernels_only:
        line["cpu_baseline"] = cpu_baseline(wl, os.cpu_count() or 1, args.cpu_seconds)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload.startswith("precision"):
        run_precision(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
