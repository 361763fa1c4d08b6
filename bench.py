#!/usr/bin/env python
"""bench.py -- decoded MPix/s of the baseline-JPEG decode path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cudajpeg|reference]
                    [--workload single_4096|single_1024]

One step = one decode of one synthetic JPEG (default: 4096x4096 4:2:0 q90,
about 2.6 MB of entropy-coded data) through the whole path: destuff, parallel
Huffman decode, coefficient write-out, fused iDCT + upsample + colour.

* ``value``   device-resident throughput: the compressed bytes are already in
  HBM when the timed region starts (cjReaderRedecodeDevice); each step is
  timed with CUDA events on the decoder's stream, and L2 is flushed (256 MiB
  write) before every step, outside the events.  Max over ranks.
* ``e2e``     the same metric through the public C API (openJPGMem): per step
  the host->device copy of the scan from pinned memory, the decode, and the
  device->host copy of the RGB image into the reader's pinned buffer.
* ``roofline`` the dominant kernel's algorithmic bytes / its mean duration
  (per-kernel CUDA events inside the timed region) against the measured HBM
  copy bandwidth in MEASURED_PEAKS.json.
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

# Algorithmic bytes of each kernel, per launch, as a function of the image:
# B = entropy-coded bytes, Bd = destuffed bytes, n = 8x8 blocks, P = output bytes.
KERNEL_BYTES = {
    "k_destuff_count": lambda g: g["B"],
    "k_scan_tiles": lambda g: 0,
    "k_destuff_scatter": lambda g: g["B"] + g["Bd"],
    "k_build_segments": lambda g: 0,
    "k_sync_intra": lambda g: g["Bd"],
    "k_sync_inter": lambda g: g["Bd"],
    "k_scan_warps": lambda g: 0,
    "k_decode_write": lambda g: g["Bd"] + 128 * g["n"],
    "k_pixel": lambda g: 128 * g["n"] + g["P"],
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cudajpeg", choices=["cudajpeg", "reference"])
    ap.add_argument("--workload", default="single_4096", choices=["single_4096", "single_1024"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def make_workload(name: str):
    from cudajpeg_b200 import workloads as W
    s = W.single_4096() if name == "single_4096" else W.single_1024()
    cfg = {"workload": f"{name}_{s.mode}_q{s.quality}", "width": s.width, "height": s.height,
           "subsampling": {"420": "4:2:0", "422": "4:2:2", "444": "4:4:4"}.get(s.mode, "grey"),
           "quality": s.quality, "restart_interval": s.restart, "file_bytes": len(s.data),
           "data": "synthetic, seeded (cudajpeg_b200/workloads.py), Pillow/libjpeg encoder with "
                   "Annex K Huffman tables"}
    return s, cfg


# ---------------------------------------------------------------- CPU baseline

def ref_cpu_time(data: bytes, threads: int, budget_s: float):
    """Time the reference CPUonly decoder (oracle/_ref) -- or, if that build
    is absent, the oracle port -- with one image per thread on `threads`
    host threads for about `budget_s` seconds.  Returns (kind, seconds,
    decoded pixels)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    d = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    fd, path = tempfile.mkstemp(suffix=".jpg", dir=d)
    with os.fdopen(fd, "wb") as f:
        f.write(data)
    try:
        if O.ref_available():
            secs, px, fails = O.ref_cpu_bench([path], 1, 1)  # calibrate: one decode
            if fails:
                raise RuntimeError("reference CPUonly decoder failed on the workload")
            iters = max(1, int(budget_s / max(secs, 1e-4)))
            secs, px, fails = O.ref_cpu_bench([path] * threads, iters, threads)
            return "reference", secs, px
        from concurrent.futures import ThreadPoolExecutor
        t0 = time.perf_counter()
        ref = O.decode(data)
        per = time.perf_counter() - t0
        iters = max(1, int(budget_s / per))
        t0 = time.perf_counter()
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(lambda _: O.decode(data), range(iters * threads)))
        return "port", time.perf_counter() - t0, iters * threads * ref.width * ref.height
    finally:
        os.unlink(path)


def cpu_baseline(sample, threads: int, budget_s: float) -> dict:
    kind, secs, px = ref_cpu_time(sample.data, threads, budget_s)
    nimg = px // sample.pixels
    who = ("reference CPUonly openJPG, CPUonly/src/main.c:10" if kind == "reference"
           else "oracle port of the reference path")
    return {"value": round(px / secs / 1e6, 3), "unit": "MPix/s", "cores": threads, "kind": kind,
            "sample": f"{nimg} decodes of the workload file from /dev/shm in {secs:.1f} s "
                      f"({who}, one image per thread)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sample, cfg = make_workload(args.workload)
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        O.build()
    # per step: every thread decodes the workload once
    d = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    fd, path = tempfile.mkstemp(suffix=".jpg", dir=d)
    with os.fdopen(fd, "wb") as f:
        f.write(sample.data)
    try:
        kind = "reference" if O.ref_available() else "port"
        times = []
        for k in range(args.warmup + args.steps):
            if kind == "reference":
                secs, px, fails = O.ref_cpu_bench([path] * threads, 1, threads)
                if fails:
                    raise RuntimeError("reference decode failed")
            else:
                from concurrent.futures import ThreadPoolExecutor
                t0 = time.perf_counter()
                with ThreadPoolExecutor(threads) as ex:
                    list(ex.map(lambda _: O.decode(sample.data), range(threads)))
                secs = time.perf_counter() - t0
            if k >= args.warmup:
                times.append(secs)
    finally:
        os.unlink(path)
    total = sum(times)
    value = threads * sample.pixels * args.steps / total / 1e6
    line = {"metric": METRIC, "value": round(value, 3), "unit": "MPix/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/int32", "data": "synthetic",
            "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": round(value, 3), "unit": "MPix/s", "cores": threads,
                             "kind": kind,
                             "sample": f"each step decodes the workload once on each of {threads} "
                                       f"threads (CPUonly openJPG from /dev/shm)"},
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


def read_traffic(kernel: str, workload: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def run_gpu(args):
    import numpy as np
    import torch

    import cudajpeg_b200 as cj

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    sample, cfg = make_workload(args.workload)
    n = len(sample.data)
    src = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    src.numpy()[:] = np.frombuffer(sample.data, np.uint8)
    reader = cj.Reader()
    reader.open_bytes((src.data_ptr(), n))
    info = reader.info()
    ext = torch.cuda.ExternalStream(reader.stream())
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    npix = sample.pixels
    out_bytes = npix * (3 if info["channels"] == 3 else 1)
    nblocks = info["mcux"] * info["mcuy"] * info["bpm"]
    geom = {"B": info["scan_bytes"], "Bd": info["destuffed"], "n": nblocks, "P": out_bytes}

    # warm-up (device-resident path, then the public API path)
    for _ in range(args.warmup):
        reader.redecode_device()
    reader.open_bytes((src.data_ptr(), n))
    torch.cuda.synchronize()
    if reader.sync():
        raise RuntimeError("warm-up decode reported an error")

    # ---- timed: device-resident decode
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
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * npix * args.steps / (total_ms / 1e3) / 1e6

    # ---- timed: end to end through openJPGMem (H2D + decode + D2H)
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
    e2e_total = sum(e2e_ms)
    if dist:
        t = torch.tensor([e2e_total], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * npix * args.steps / (e2e_total / 1e3) / 1e6
    lat = sorted(e2e_ms)

    # ---- roofline of the dominant kernel
    means = {k: statistics.mean(v) for k, v in kern_ms.items()}
    dom = max(means, key=means.get)
    peaks = read_peaks()
    alg = KERNEL_BYTES[dom](geom)
    achieved = alg / (means[dom] / 1e3) / 1e9
    traffic = read_traffic(dom, args.workload)
    kshare = {k: round(v / sum(means.values()), 4) for k, v in means.items()}

    line = {"metric": METRIC, "value": round(value, 2), "unit": "MPix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8/int16/int32", "data": "synthetic",
            "config": dict(cfg, parallelism=f"replicas{world}",
                           l2="flushed before each step (256 MiB write, outside the timing)",
                           compressed_MB_per_s=round(world * info["scan_bytes"] * args.steps
                                                     / (total_ms / 1e3) / 1e6, 1)),
            "e2e": {"value": round(e2e_value, 2), "unit": "MPix/s",
                    "h2d_bytes_per_step": info["scan_bytes"] + info["param_bytes"],
                    "d2h_bytes_per_step": out_bytes + 32,
                    "latency_ms_p50": round(lat[len(lat) // 2], 3),
                    "latency_ms_p99": round(lat[min(len(lat) - 1, int(0.99 * len(lat)))], 3)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4),
                         "traffic": traffic, "algorithmic_bytes": int(alg),
                         "peak_source": peaks["source"]},
            "kernel_ms": {k: round(v, 4) for k, v in means.items()}, "kernel_share": kshare,
            "gpu_launches": int(launches),
            "clocks": clocks.summary()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sample, os.cpu_count() or 1, args.cpu_seconds)
    reader.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
