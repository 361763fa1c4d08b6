"""Seeded synthetic baseline JPEGs for the decode workloads.

There is no public dataset behind the reference's numbers: these generators
*are* the benchmark inputs.  Every image is drawn from a seed, encoded by
Pillow's libjpeg with ``optimize=False`` (the ITU T.81 Annex K Huffman
tables), ``quality=`` (IJG-scaled Annex K quantisation tables), ``subsampling=``
(0 = 4:4:4, 1 = 4:2:2, 2 = 4:2:0) and ``restart_marker_blocks=`` (a DRI
interval in MCUs).  Grey images are single-component.

Workloads (sizes and value distributions follow the benchmark configurations):

* ``single_1024``  -- 1024x768 4:2:0 q75, smooth sinusoid/gradient + N(0, 8)
* ``single_4096``  -- 4096x4096 4:2:0 q90, 8 random-orientation sinusoids plus
  uniform luma noise; the noise is U(+-5) rather than U(+-16) so that the
  entropy data lands at the 2-3 MB the workload is specified at (U(+-16)
  gives 5.9 MB at q90)
* ``precision_8192`` -- 8192x8192 q95, 50/50 U(0,255) noise and a gradient,
  in 4:4:4, 4:2:2 and grey
* ``mixed_batch``  -- N images, W and H log-uniform in [64, 2048] (multiples of
  8), 4:2:0/4:2:2/4:4:4/grey with p = .6/.2/.1/.1, q ~ U[50, 95], 30% with a
  restart interval of 16-64 MCUs, content as ``single_1024``
"""
from __future__ import annotations

import io
from dataclasses import dataclass

import numpy as np

SUBSAMPLING = {"444": 0, "422": 1, "420": 2}


@dataclass
class JpegSample:
    data: bytes
    width: int
    height: int
    mode: str          # "420" | "422" | "444" | "gray"
    quality: int
    restart: int       # DRI interval in MCUs (0 = none)

    @property
    def pixels(self) -> int:
        return self.width * self.height


def encode(arr: np.ndarray, mode: str, quality: int, restart: int = 0,
           optimize: bool = False) -> bytes:
    """Encode uint8 [H,W,3] (colour) or [H,W] (grey) as a baseline JPEG."""
    from PIL import Image

    buf = io.BytesIO()
    kw = dict(quality=int(quality), optimize=optimize, progressive=False)
    if restart:
        kw["restart_marker_blocks"] = int(restart)
    if mode == "gray":
        img = Image.fromarray(arr if arr.ndim == 2 else arr[..., 0], "L")
    else:
        img = Image.fromarray(arr, "RGB")
        kw["subsampling"] = SUBSAMPLING[mode]
    # (optimize=True fails inside Pillow when the compressed scan outgrows
    # the encoder buffer it sizes from the pixel count: near-incompressible
    # content at quality >= 95)
    img.save(buf, "JPEG", **kw)
    return buf.getvalue()


def smooth_content(rng: np.random.Generator, w: int, h: int, channels: int) -> np.ndarray:
    """Smooth 2-D sinusoid/gradient field + Gaussian noise (sigma 8), clipped."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    out = np.empty((h, w, channels), np.uint8)
    for c in range(channels):
        fx, fy = rng.uniform(0.5, 4.0, 2) * 2 * np.pi / np.array([w, h])
        ph = rng.uniform(0, 2 * np.pi, 2)
        gx, gy = rng.uniform(-60, 60, 2)
        f = (128 + 70 * np.sin(fx * x + ph[0]) * np.cos(fy * y + ph[1])
             + gx * (x / w - 0.5) + gy * (y / h - 0.5))
        f += rng.normal(0, 8, (h, w)).astype(np.float32)
        out[..., c] = np.clip(f, 0, 255).astype(np.uint8)
    return out


def texture_content(rng: np.random.Generator, w: int, h: int, amp: float = 11.0,
                    noise: float = 16.0) -> np.ndarray:
    """Sum of 8 random-orientation sinusoids + uniform noise +-``noise``."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    out = np.empty((h, w, 3), np.uint8)
    base = np.zeros((h, w), np.float32)
    for _ in range(8):
        th = rng.uniform(0, np.pi)
        k = rng.uniform(2, 40) * 2 * np.pi / max(w, h)
        base += amp * np.sin(k * (np.cos(th) * x + np.sin(th) * y) + rng.uniform(0, 2 * np.pi))
    # the noise is shared by R, G and B (a luma texture); the colour channels
    # differ by a slow tint so chroma stays smooth
    shared = rng.uniform(-noise, noise, (h, w)).astype(np.float32)
    for c in range(3):
        tint = rng.uniform(-30, 30) * (x / w - 0.5)
        out[..., c] = np.clip(128 + base + shared + tint, 0, 255).astype(np.uint8)
    return out


def noise_gradient_content(rng: np.random.Generator, w: int, h: int, channels: int) -> np.ndarray:
    """50/50 blend of white noise U(0,255) and a smooth gradient."""
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    out = np.empty((h, w, channels), np.uint8)
    for c in range(channels):
        grad = 255 * (0.5 * x / w + 0.5 * y / h)
        if c:
            grad = 255 - grad
        noise = rng.integers(0, 256, (h, w), dtype=np.uint8).astype(np.float32)
        out[..., c] = np.clip(0.5 * noise + 0.5 * grad, 0, 255).astype(np.uint8)
    return out


def single_1024(seed: int = 1) -> JpegSample:
    rng = np.random.default_rng(seed)
    arr = smooth_content(rng, 1024, 768, 3)
    return JpegSample(encode(arr, "420", 75), 1024, 768, "420", 75, 0)


def single_4096(seed: int = 2) -> JpegSample:
    rng = np.random.default_rng(seed)
    arr = texture_content(rng, 4096, 4096, noise=5.0)
    return JpegSample(encode(arr, "420", 90), 4096, 4096, "420", 90, 0)


def precision_8192(mode: str, seed: int = 3, size: int = 8192) -> JpegSample:
    rng = np.random.default_rng(seed)
    ch = 1 if mode == "gray" else 3
    arr = noise_gradient_content(rng, size, size, ch)
    return JpegSample(encode(arr if ch == 3 else arr[..., 0], mode, 95), size, size, mode, 95, 0)


def _mixed_one(args) -> JpegSample:
    seed, k, w, h, mode, q, ri = args
    rng = np.random.default_rng([seed, k])
    arr = smooth_content(rng, w, h, 1 if mode == "gray" else 3)
    return JpegSample(encode(arr if mode != "gray" else arr[..., 0], mode, q, ri), w, h, mode, q, ri)


def mixed_batch_plan(n: int = 1024, seed: int = 4, max_side: int = 2048) -> list:
    """Per-image (seed, index, w, h, mode, quality, restart) of a mixed batch."""
    rng = np.random.default_rng(seed)
    modes = np.array(["420", "422", "444", "gray"])
    plan = []
    for k in range(n):
        w, h = (np.exp(rng.uniform(np.log(64), np.log(max_side), 2)) / 8).round().astype(int) * 8
        w, h = int(max(w, 8)), int(max(h, 8))
        mode = str(rng.choice(modes, p=[0.6, 0.2, 0.1, 0.1]))
        q = int(rng.integers(50, 96))
        ri = int(rng.integers(16, 65)) if rng.random() < 0.3 else 0
        plan.append((seed, k, w, h, mode, q, ri))
    return plan


def mixed_batch(n: int = 1024, seed: int = 4, max_side: int = 2048, workers: int = 0) -> list:
    """The mixed batch; `workers` > 1 encodes in a spawn-started process pool
    (safe to call after CUDA has been initialised)."""
    plan = mixed_batch_plan(n, seed, max_side)
    if workers and workers > 1 and n > 8:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            return list(ex.map(_mixed_one, plan, chunksize=8))
    return [_mixed_one(a) for a in plan]


def small_case(seed: int, w: int, h: int, mode: str, quality: int = 85, restart: int = 0,
               content: str = "smooth", optimize: bool = False) -> JpegSample:
    """A small seeded image for parity tests."""
    rng = np.random.default_rng(seed)
    ch = 1 if mode == "gray" else 3
    if content == "noise":
        arr = noise_gradient_content(rng, w, h, ch)
    elif content == "texture" and ch == 3:
        arr = texture_content(rng, w, h)
    else:
        arr = smooth_content(rng, w, h, ch)
    if ch == 1:
        arr = arr[..., 0]
    return JpegSample(encode(arr, mode, quality, restart, optimize), w, h, mode, quality, restart)
