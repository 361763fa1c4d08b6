"""Continuous-batching decode server (include/cudajpeg.h cjServer*).

The reference decodes one file per process (src/main.cu); this is the
serving form built on the batch decoder.  Requests are single JPEGs; the
native worker thread admits waiting requests into free batch engines while
the projected device bytes of the batches in flight stay within a budget,
so requests that arrive while others are on the GPU join the next batch.

    import cudajpeg_b200.serve as sv
    with sv.Server(engines=3) as s:
        t = s.submit(jpeg_bytes)
        res = s.wait(t)              # dict: error, width, height, channels, latency_ms
        rgb = s.copy_out(t)          # H x W x 3 (or H x W) uint8
        s.release(t)

``replay`` drives an open-loop Poisson request stream through the native
load replayer and returns latency percentiles and sustained MPix/s.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import PROGRAMMER_ERROR, DecodeError, DLPackView, load


class _Result(C.Structure):
    _fields_ = [("error", C.c_int), ("width", C.c_int), ("height", C.c_int), ("channels", C.c_int),
                ("device_pixels", C.c_void_p), ("latency_ms", C.c_double)]


STAT_KEYS = ["batches", "images", "max_batches_in_flight", "largest_batch", "waiting",
             "bytes_in_flight"]


class Server:
    def __init__(self, engines: int = 3, hbm_budget_bytes: int = 8 << 30, max_batch: int = 256):
        self.lib = load()
        self.ptr = self.lib.cjServerCreate(engines, hbm_budget_bytes, max_batch)
        if not self.ptr:
            raise RuntimeError("cjServerCreate failed (no CUDA device?)")

    def close(self):
        if self.ptr:
            self.lib.cjServerDestroy(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, jpeg: bytes) -> int:
        t = self.lib.cjServerSubmit(self.ptr, jpeg, len(jpeg))
        if t < 0:
            raise DecodeError(int(-t) if t < -1 else int(t), "cjServerSubmit")
        return int(t)

    def wait(self, ticket: int, timeout_s: float = 60.0) -> dict:
        r = _Result()
        rc = self.lib.cjServerWait(self.ptr, ticket, timeout_s, C.byref(r))
        if rc == 1:
            raise TimeoutError(f"request {ticket} not finished after {timeout_s} s")
        if rc:
            raise DecodeError(rc, f"cjServerWait({ticket})")
        return {"error": r.error, "width": r.width, "height": r.height, "channels": r.channels,
                "device_pixels": r.device_pixels, "latency_ms": r.latency_ms}

    def copy_out(self, ticket: int, res: dict | None = None) -> np.ndarray:
        res = res or self.wait(ticket)
        if res["error"]:
            raise DecodeError(res["error"], f"request {ticket}")
        h, w, c = res["height"], res["width"], res["channels"]
        out = np.empty((h, w, 3) if c == 3 else (h, w), np.uint8)
        rc = self.lib.cjServerCopyOut(self.ptr, ticket, out.ctypes.data, out.nbytes)
        if rc:
            raise DecodeError(rc, f"cjServerCopyOut({ticket})")
        return out

    def device_tensor(self, ticket: int):
        """A finished request's pixels as a torch tensor on the GPU, without
        a copy (cjServerDLPack); valid until release(ticket)."""
        import torch
        p = self.lib.cjServerDLPack(self.ptr, ticket)
        if not p:
            raise DecodeError(PROGRAMMER_ERROR, f"request {ticket} has no device pixels")
        return torch.from_dlpack(DLPackView(p, self.lib))

    def set_tuning(self, sub_bits: int = 0, decode_ctas_per_sm: int = 0, pixel_tile_cap: int = 0):
        err = self.lib.cjServerSetTuning(self.ptr, sub_bits, decode_ctas_per_sm, pixel_tile_cap)
        if err:
            raise ValueError(f"bad tuning {(sub_bits, decode_ctas_per_sm, pixel_tile_cap)}")

    def release(self, ticket: int):
        self.lib.cjServerRelease(self.ptr, ticket)

    def stats(self) -> dict:
        a = (C.c_longlong * 6)()
        self.lib.cjServerStats(self.ptr, a)
        return dict(zip(STAT_KEYS, [int(v) for v in a]))

    def replay(self, files: list, arrival_s: np.ndarray) -> dict:
        """Open-loop replay: request k is files[k % len(files)], submitted at
        arrival_s[k] seconds.  Returns latencies (ms, scheduled arrival ->
        batch done on the GPU), per-request errors and the wall time."""
        sizes = np.array([len(f) for f in files], np.int64)
        offsets = np.zeros(len(files), np.int64)
        offsets[1:] = np.cumsum(sizes)[:-1]
        blob = np.frombuffer(b"".join(files), np.uint8)
        arrival_s = np.ascontiguousarray(arrival_s, np.float64)
        n = len(arrival_s)
        lat = np.zeros(n, np.float64)
        errs = np.zeros(n, np.int32)
        wall = C.c_double(0.0)
        rc = self.lib.cjServerReplay(self.ptr, blob.ctypes.data, offsets.ctypes.data, sizes.ctypes.data,
                                     len(files), arrival_s.ctypes.data, n, lat.ctypes.data,
                                     errs.ctypes.data, C.byref(wall))
        if rc:
            raise DecodeError(rc, "cjServerReplay")
        return {"latency_ms": lat, "errors": errs, "wall_s": wall.value}


def poisson_arrivals(rate: float, n: int, seed: int = 0) -> np.ndarray:
    """Arrival times (s) of an open-loop Poisson stream of `rate` requests/s."""
    rng = np.random.default_rng([seed, int(rate)])
    return np.cumsum(rng.exponential(1.0 / rate, n))


def summarize(run: dict, pixels: np.ndarray, rate: float) -> dict:
    """p50/p99/p99.9 latency and sustained MPix/s of one replay; `pixels[k]`
    is the pixel count of file k (requests cycle through the files)."""
    lat = run["latency_ms"]
    n = len(lat)
    px = pixels[np.arange(n) % len(pixels)].sum()
    return {
        "offered_img_s": rate,
        "requests": n,
        "errors": int(np.count_nonzero(run["errors"])),
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "p999_ms": float(np.percentile(lat, 99.9)),
        "achieved_img_s": n / run["wall_s"],
        "mpix_s": px / run["wall_s"] / 1e6,
    }
