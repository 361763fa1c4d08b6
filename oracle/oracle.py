"""ctypes front end of the CPU checker.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module; the decoder in ``cudajpeg_b200`` never does.

Three libraries sit behind it (all built by ``oracle/Makefile``):

* ``liboracle.so`` -- our C restatement of the reference path
  (``jpeg_oracle.c``; see its header for the reference file:line map);
* ``_ref/libref_cpuonly.so`` -- the reference's own CPUonly decoder compiled
  from its sources: the pixel oracle and the timed CPU baseline;
* ``_ref/libref_gputree.so`` -- the reference's ``src/format.cu`` +
  ``src/decodeScanCPU.cu`` built as host C++: the coefficient oracle, which
  also decodes restart-marker files.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

ERROR_NAMES = {0: "NO_ERROR", 1: "SYNTAX_ERROR", 2: "UNSUPPORTED_ERROR", 3: "OOM_ERROR",
               4: "CUDA_MEM_ERROR", 5: "FILE_ERROR", 6: "CUDA_KERNEL_LAUNCH_ERROR",
               -1: "PROGRAMMER_ERROR"}

_lib = None
_ref_cpu = None
_ref_gpu = None


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.oracle_decode.restype = C.c_void_p
        lib.oracle_decode.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_int)]
        lib.oracle_free.argtypes = [C.c_void_p]
        lib.oracle_info.argtypes = [C.c_void_p, C.c_void_p]
        lib.oracle_coefs.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.oracle_plane.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.oracle_pixels.argtypes = [C.c_void_p, C.c_void_p]
        lib.oracle_dq.argtypes = [C.c_void_p, C.c_void_p]
        lib.oracle_idct_blocks.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        lib.oracle_idct_f64.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        lib.oracle_fancy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_fancy_upsample.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                              C.c_void_p, C.c_int, C.c_int]
        _lib = lib
    return _lib


@dataclass
class Component:
    samples_x: int
    samples_y: int
    width: int
    height: int
    stride: int
    rows: int
    nblocks: int
    dq_id: int


@dataclass
class Decoded:
    error: int
    width: int = 0
    height: int = 0
    nch: int = 0
    mcux: int = 0
    mcuy: int = 0
    restart_interval: int = 0
    comps: list = field(default_factory=list)
    coefs: list = field(default_factory=list)   # int32 [nblocks, 64] per component
    planes: list = field(default_factory=list)  # uint8 [rows, stride] per component
    pixels: np.ndarray | None = None            # uint8 [H, W, 3] or [H, W]
    dq: np.ndarray | None = None                # uint16 [4, 64] zig-zag order
    fancy_ycc: np.ndarray | None = None         # uint8 [H, W, 3], fancy=True only
    fancy_rgb: np.ndarray | None = None         # uint8 [H, W, 3], fancy=True only


def decode(data: bytes, fancy: bool = False) -> Decoded:
    """Decode a JPEG held in memory with the C restatement.  fancy=True also
    gives colour images with fancy (triangle) chroma upsampling: upsampled
    YCbCr and RGB through the reference's colour transform."""
    lib = _load()
    err = C.c_int(0)
    h = lib.oracle_decode(data, len(data), C.byref(err))
    try:
        out = Decoded(error=err.value)
        if err.value != 0 or not h:
            return out
        info = np.zeros(6 + 8 * 3, np.int32)
        lib.oracle_info(h, info.ctypes.data)
        out.width, out.height, out.nch, out.mcux, out.mcuy, out.restart_interval = map(int, info[:6])
        for c in range(out.nch):
            comp = Component(*map(int, info[6 + 8 * c: 14 + 8 * c]))
            out.comps.append(comp)
            coef = np.empty((comp.nblocks, 64), np.int32)
            lib.oracle_coefs(h, c, coef.ctypes.data)
            plane = np.empty((comp.rows, comp.stride), np.uint8)
            lib.oracle_plane(h, c, plane.ctypes.data)
            out.coefs.append(coef)
            out.planes.append(plane)
        shape = (out.height, out.width, 3) if out.nch == 3 else (out.height, out.width)
        out.pixels = np.empty(shape, np.uint8)
        lib.oracle_pixels(h, out.pixels.ctypes.data)
        out.dq = np.empty((4, 64), np.uint16)
        lib.oracle_dq(h, out.dq.ctypes.data)
        if fancy and out.nch == 3:
            out.fancy_ycc = np.empty((out.height, out.width, 3), np.uint8)
            out.fancy_rgb = np.empty((out.height, out.width, 3), np.uint8)
            lib.oracle_fancy(h, out.fancy_ycc.ctypes.data, out.fancy_rgb.ctypes.data)
        return out
    finally:
        if h:
            lib.oracle_free(h)


def fancy_upsample(plane: np.ndarray, xs: int, ys: int, ow: int, oh: int) -> np.ndarray:
    """Fancy (triangle) upsampling of a 2-D uint8 plane by 2^xs x 2^ys,
    cropped to oh x ow (oracle_fancy_upsample)."""
    lib = _load()
    p = np.ascontiguousarray(plane, np.uint8)
    out = np.empty((oh, ow), np.uint8)
    lib.oracle_fancy_upsample(p.ctypes.data, p.shape[1], p.shape[0], p.shape[1], xs, ys, out.ctypes.data, ow, oh)
    return out


def idct_int(coefs: np.ndarray) -> np.ndarray:
    """Reference integer iDCT of int32 natural-order blocks -> uint8 [n, 64]."""
    lib = _load()
    c = np.ascontiguousarray(coefs, np.int32).reshape(-1, 64)
    out = np.empty(c.shape, np.uint8)
    lib.oracle_idct_blocks(c.ctypes.data, c.shape[0], out.ctypes.data)
    return out


def idct_f64(coefs: np.ndarray) -> np.ndarray:
    """Exact FP64 iDCT (before +128, rounding and clip) -> float64 [n, 64]."""
    lib = _load()
    c = np.ascontiguousarray(coefs, np.int32).reshape(-1, 64)
    out = np.empty(c.shape, np.float64)
    lib.oracle_idct_f64(c.ctypes.data, c.shape[0], out.ctypes.data)
    return out


def quantised(d: Decoded) -> list:
    """Per-component quantised coefficients (dequantised // Q), int32 [n, 64]."""
    zz = np.array([0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48,
                   41, 34, 27, 20, 13, 6, 7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15,
                   23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63])
    out = []
    for comp, coef in zip(d.comps, d.coefs):
        q = np.zeros(64, np.int64)
        q[zz] = d.dq[comp.dq_id]
        q[q == 0] = 1
        out.append((coef // q).astype(np.int32))
    return out


# ---------------------------------------------------------------- reference builds

def ref_available() -> bool:
    return (os.path.exists(os.path.join(REF_DIR, "libref_cpuonly.so"))
            and os.path.exists(os.path.join(REF_DIR, "libref_gputree.so")))


def _load_ref():
    global _ref_cpu, _ref_gpu
    if _ref_cpu is None:
        cpu = C.CDLL(os.path.join(REF_DIR, "libref_cpuonly.so"))
        cpu.refcpu_open.restype = C.c_void_p
        cpu.refcpu_open.argtypes = [C.c_char_p]
        cpu.refcpu_info.argtypes = [C.c_void_p, C.c_void_p]
        cpu.refcpu_pixels.argtypes = [C.c_void_p, C.c_void_p]
        cpu.refcpu_close.argtypes = [C.c_void_p]
        cpu.refcpu_open_any.restype = C.c_void_p
        cpu.refcpu_open_any.argtypes = [C.c_char_p]
        cpu.refcpu_use_gputree.argtypes = [C.c_char_p]
        cpu.refcpu_bench.restype = C.c_double
        cpu.refcpu_bench.argtypes = [C.POINTER(C.c_char_p), C.c_int, C.c_int, C.c_int,
                                     C.POINTER(C.c_longlong), C.POINTER(C.c_int)]
        gpu = C.CDLL(os.path.join(REF_DIR, "libref_gputree.so"))
        gpu.refgpu_new.restype = C.c_void_p
        gpu.refgpu_del.argtypes = [C.c_void_p]
        gpu.refgpu_open.argtypes = [C.c_void_p, C.c_char_p]
        gpu.refgpu_info.argtypes = [C.c_void_p, C.c_void_p]
        gpu.refgpu_coefs.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        # restart-marker files, which CPUonly rejects, through the reference's
        # GPU-tree coefficient decoder + CPUonly's iDCT and colour stage
        if not cpu.refcpu_use_gputree(os.path.join(REF_DIR, "libref_gputree.so").encode()):
            raise OSError("libref_gputree.so could not be loaded into the CPUonly harness")
        _ref_cpu, _ref_gpu = cpu, gpu
    return _ref_cpu, _ref_gpu


class _QuietStdout:
    """The reference decoders printf diagnostics to stdout (e.g.
    CPUonly/src/decodeScanCPU.c:41,152); route fd 1 to /dev/null meanwhile."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        C.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def ref_cpu_pixels(path: str, restart: bool = False):
    """Reference CPUonly decode of a file -> pixels array, or None on failure.
    restart=True: a file CPUonly rejects (restart markers) goes through the
    reference's GPU-tree coefficient decoder (src/decodeScanCPU.cu:98-152)
    and CPUonly's iDCT and colour stage instead."""
    cpu, _ = _load_ref()
    with _QuietStdout():
        h = (cpu.refcpu_open_any if restart else cpu.refcpu_open)(path.encode())
    if not h:
        return None
    try:
        info = np.zeros(4, np.int32)
        cpu.refcpu_info(h, info.ctypes.data)
        w, hgt, nch = map(int, info[:3])
        shape = (hgt, w, 3) if nch == 3 else (hgt, w)
        px = np.empty(shape, np.uint8)
        cpu.refcpu_pixels(h, px.ctypes.data)
        return px
    finally:
        cpu.refcpu_close(h)


def ref_gpu_coefs(path: str):
    """Reference GPU-tree host decode -> (error, [int32 [n,64] per component])."""
    _, gpu = _load_ref()
    r = gpu.refgpu_new()
    try:
        with _QuietStdout():
            err = gpu.refgpu_open(r, path.encode())
        if err:
            return err, []
        info = np.zeros(18, np.int32)
        gpu.refgpu_info(r, info.ctypes.data)
        out = []
        for c in range(int(info[2])):
            n = int(info[8 + 4 * c])
            a = np.empty(n, np.int32)
            gpu.refgpu_coefs(r, c, a.ctypes.data)
            out.append(a.reshape(-1, 64))
        return 0, out
    finally:
        gpu.refgpu_del(r)


def ref_cpu_bench(paths, iters: int, threads: int):
    """Time the reference CPUonly decoder -- restart-marker files through the
    GPU-tree coefficient decoder + CPUonly pixel stage -- : (seconds, pixels,
    failures)."""
    cpu, _ = _load_ref()
    arr = (C.c_char_p * len(paths))(*[p.encode() for p in paths])
    px = C.c_longlong(0)
    fails = C.c_int(0)
    with _QuietStdout():
        secs = cpu.refcpu_bench(arr, len(paths), iters, threads, C.byref(px), C.byref(fails))
    return secs, px.value, fails.value
