"""cudajpeg_b200 -- B200-native baseline-JPEG decoder.

The decoder is ``libcudajpeg.so`` (C ABI in ``include/*.h``, CUDA kernels for
sm_100a in ``csrc/``); this package builds it in-tree and binds it with
ctypes.  There is no CPU decode path: without the library or a GPU every
call fails with an exception.

    import cudajpeg_b200 as cj
    with cj.Reader() as r:
        r.open("image.jpg")          # openJPG
        rgb = r.pixels()             # H x W x 3 uint8 (H x W for grey)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcudajpeg.so")

# format.h error codes
NO_ERROR = 0
SYNTAX_ERROR = 1
UNSUPPORTED_ERROR = 2
OOM_ERROR = 3
CUDA_MEM_ERROR = 4
FILE_ERROR = 5
CUDA_KERNEL_LAUNCH_ERROR = 6
PROGRAMMER_ERROR = -1
ERROR_NAMES = {0: "NO_ERROR", 1: "SYNTAX_ERROR", 2: "UNSUPPORTED_ERROR", 3: "OOM_ERROR",
               4: "CUDA_MEM_ERROR", 5: "FILE_ERROR", 6: "CUDA_KERNEL_LAUNCH_ERROR",
               -1: "PROGRAMMER_ERROR"}

READER_HOST_COEFFICIENTS = 1
IDCT_INT, IDCT_F32, IDCT_TC = 0, 1, 2
OUTPUT_RGB, OUTPUT_PLANAR, OUTPUT_NV12, OUTPUT_RGB_FANCY = 0, 1, 2, 3
# chroma sampling classes (per-class subsequence sizes)
SAMPLING_420, SAMPLING_422, SAMPLING_444, SAMPLING_GRAY, SAMPLING_OTHER = 0, 1, 2, 3, 4
SAMPLING_CLASSES = 5

# Every symbol the C headers in include/ declare (checked by the CPU tests).
EXPORTED = [
    "read16", "delJPGReader", "newJPGReader", "openJPG", "openJPGMem", "writeJPG",
    "printError", "skipBlock", "decodeSOF", "decodeDHT", "decodeDQT", "decodeDRI",
    "decodeScanGPU", "iDCT_resample_colourTransform", "cjIDCTPlane", "cjIDCTBlocksRaw",
    "cjReaderInfo", "cjReaderPixels", "cjReaderSetFlags", "cjReaderSetSubsequenceBits",
    "cjReaderStageTimes", "cjReaderDeviceCoefficients", "cjReaderDeviceQuantTable",
    "cjReaderStream", "cjDebugHuffDecode", "cjReaderRedecodeDevice", "cjReaderSync",
    "cjReaderDevicePixels", "cjReaderSetProfile", "cjReaderKernelTimes", "cjReaderLaunchCount",
    "cjBatchCreate", "cjBatchDestroy", "cjBatchSetSubsequenceBits", "cjBatchStage", "cjBatchRun",
    "cjBatchFetch", "cjBatchWait", "cjBatchDecode", "cjBatchImage", "cjBatchDeviceImage",
    "cjBatchStream", "cjBatchStats", "cjBatchKernelMs", "cjBatchPhaseTimes",
    "cjDecodeNoAlloc", "cjBatchImageGeometry",
    "cjServerCreate", "cjServerDestroy", "cjServerSubmit", "cjServerWait", "cjServerCopyOut",
    "cjServerRelease", "cjServerStats", "cjServerReplay", "cjServerSetTuning",
    "cjBatchSetTuning", "cjBatchGetTuning", "cjBatchAutotune", "cjDebugStepTable",
    "cjBatchCopyCoefficients", "cjBuildInfo", "cjBatchSetWaitLimit", "cjBatchSetOutput",
    "cjBatchSetSubsequenceBitsFor", "cjBatchGetSubsequenceBitsFor",
    "cjBatchGetOutput", "cjBatchChromaGeometry", "cjBatchDLPack", "cjServerDLPack", "cjDLPackFree",
    "decodeScanCPU", "upsampleAndColourTransformHybrid", "upsampleAndColourTransformGPU",
    "upsampleAndColourTransformCPU", "cjBatchSetParse", "cjDebugParseCompare", "cjBatchSetHypotheses",
]

BATCH_PHASES = ["tables", "destuff_count", "tile_scan", "destuff_scatter", "segments", "sync",
                "fixup", "warp_scan", "write", "pixel", "launch"]

KERNEL_NAMES = ["k_decode_batch", "k_pixel", "k_prog_scan"]


class DecodeError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{ERROR_NAMES.get(code, code)}{': ' + what if what else ''}")


_lib = None


def load(build_if_missing: bool = True):
    """Load libcudajpeg.so (building it with nvcc if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise OSError(f"{LIB_PATH} is not built (python -m cudajpeg_b200.build)")
        from . import build as _build
        _build.build()
    lib = C.CDLL(LIB_PATH)
    vp, i64p = C.c_void_p, C.POINTER(C.c_int64)
    lib.newJPGReader.restype = vp
    lib.delJPGReader.argtypes = [vp]
    lib.openJPG.argtypes = [vp, C.c_char_p]
    lib.openJPGMem.argtypes = [vp, vp, C.c_size_t]
    lib.writeJPG.argtypes = [vp, C.c_char_p]
    lib.printError.argtypes = [vp]
    lib.read16.restype = C.c_ushort
    lib.read16.argtypes = [vp]
    lib.cjReaderInfo.argtypes = [vp, i64p]
    lib.cjReaderPixels.restype = vp
    lib.cjReaderPixels.argtypes = [vp]
    lib.cjReaderSetFlags.argtypes = [vp, C.c_int]
    lib.cjReaderSetSubsequenceBits.argtypes = [vp, C.c_int]
    lib.cjReaderStageTimes.argtypes = [vp, C.POINTER(C.c_float)]
    lib.cjReaderDeviceCoefficients.restype = vp
    lib.cjReaderDeviceCoefficients.argtypes = [vp, i64p]
    lib.cjReaderDeviceQuantTable.restype = vp
    lib.cjReaderDeviceQuantTable.argtypes = [vp, C.c_int]
    lib.cjReaderStream.restype = vp
    lib.cjReaderStream.argtypes = [vp]
    lib.cjIDCTPlane.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp,
                                C.c_int, C.c_int, vp]
    lib.cjIDCTBlocksRaw.argtypes = [vp, C.c_longlong, vp, vp, C.c_int, vp]
    lib.cjDebugHuffDecode.argtypes = [vp, vp, C.c_uint]
    lib.cjDebugStepTable.argtypes = [vp, vp, C.c_int, vp]
    lib.cjBuildInfo.argtypes = [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
    lib.cjReaderRedecodeDevice.argtypes = [vp]
    lib.cjReaderSync.argtypes = [vp]
    lib.cjReaderDevicePixels.restype = vp
    lib.cjReaderDevicePixels.argtypes = [vp]
    lib.cjReaderSetProfile.argtypes = [vp, C.c_int]
    lib.cjReaderKernelTimes.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int]
    lib.cjReaderLaunchCount.restype = C.c_longlong
    lib.cjReaderLaunchCount.argtypes = [vp]
    lib.cjBatchCreate.restype = vp
    lib.cjBatchDestroy.argtypes = [vp]
    lib.cjBatchSetSubsequenceBits.argtypes = [vp, C.c_int]
    lib.cjBatchStage.argtypes = [vp, C.c_int, vp, vp, vp]
    lib.cjBatchRun.argtypes = [vp]
    lib.cjBatchFetch.argtypes = [vp]
    lib.cjBatchWait.argtypes = [vp, vp]
    lib.cjBatchDecode.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    lib.cjBatchImage.restype = vp
    lib.cjBatchImage.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]
    lib.cjBatchDeviceImage.restype = vp
    lib.cjBatchDeviceImage.argtypes = [vp, C.c_int]
    lib.cjBatchStream.restype = vp
    lib.cjBatchStream.argtypes = [vp]
    lib.cjBatchCopyCoefficients.restype = C.c_longlong
    lib.cjBatchCopyCoefficients.argtypes = [vp, C.c_int, vp, C.c_longlong]
    lib.cjBatchStats.argtypes = [vp, i64p]
    lib.cjBatchKernelMs.restype = C.c_float
    lib.cjBatchKernelMs.argtypes = [vp]
    lib.cjBatchPhaseTimes.argtypes = [vp, C.POINTER(C.c_float)]
    ip = C.POINTER(C.c_int)
    lib.cjDecodeNoAlloc.argtypes = [vp, C.c_size_t, vp, C.c_size_t, ip, ip, ip, vp]
    lib.cjBatchImageGeometry.argtypes = [vp, C.c_int, ip, ip, ip]
    lib.cjBatchSetTuning.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.cjBatchSetWaitLimit.argtypes = [vp, C.c_uint]
    lib.cjBatchSetSubsequenceBitsFor.argtypes = [vp, C.c_int, C.c_int]
    lib.cjBatchGetSubsequenceBitsFor.argtypes = [vp, C.c_int]
    lib.cjBatchSetOutput.argtypes = [vp, C.c_int, C.c_int]
    lib.cjBatchSetParse.argtypes = [vp, C.c_int]
    lib.cjBatchSetHypotheses.argtypes = [vp, C.c_int]
    lib.cjDebugParseCompare.argtypes = [vp, C.c_size_t, ip, ip]
    lib.cjBatchGetOutput.argtypes = [vp, ip, ip]
    lib.cjBatchChromaGeometry.argtypes = [vp, C.c_int, ip, ip]
    lib.cjBatchDLPack.restype = vp
    lib.cjBatchDLPack.argtypes = [vp, C.c_int]
    lib.cjServerDLPack.restype = vp
    lib.cjServerDLPack.argtypes = [vp, C.c_longlong]
    lib.cjDLPackFree.argtypes = [vp]
    lib.cjBatchGetTuning.argtypes = [vp, ip, ip, ip]
    lib.cjBatchAutotune.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, C.POINTER(C.c_float),
                                    C.POINTER(C.c_float), C.c_int]
    lib.cjServerSetTuning.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.cjServerCreate.restype = vp
    lib.cjServerCreate.argtypes = [C.c_int, C.c_longlong, C.c_int]
    lib.cjServerDestroy.argtypes = [vp]
    lib.cjServerSubmit.restype = C.c_longlong
    lib.cjServerSubmit.argtypes = [vp, vp, C.c_size_t]
    lib.cjServerWait.argtypes = [vp, C.c_longlong, C.c_double, vp]
    lib.cjServerCopyOut.argtypes = [vp, C.c_longlong, vp, C.c_size_t]
    lib.cjServerRelease.argtypes = [vp, C.c_longlong]
    lib.cjServerStats.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.cjServerReplay.argtypes = [vp, vp, vp, vp, C.c_int, vp, C.c_int, vp, vp,
                                   C.POINTER(C.c_double)]
    _lib = lib
    return lib


class Reader:
    """A JPGReader (format.h): one decoder with its own CUDA stream and
    grow-only device / pinned buffers, reused across images."""

    def __init__(self, sub_bits: int = 0, host_coefficients: bool = False):
        self.lib = load()
        self.ptr = self.lib.newJPGReader()
        if not self.ptr:
            raise MemoryError("newJPGReader failed")
        if sub_bits:
            self.set_subsequence_bits(sub_bits)
        if host_coefficients:
            self.lib.cjReaderSetFlags(self.ptr, READER_HOST_COEFFICIENTS)
        self._pinned_src = None

    def close(self):
        if self.ptr:
            self.lib.delJPGReader(self.ptr)
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

    def set_subsequence_bits(self, bits: int):
        if self.lib.cjReaderSetSubsequenceBits(self.ptr, bits):
            raise ValueError(f"bad subsequence size {bits}")

    # ---- decode
    def open(self, path: str, check: bool = True) -> int:
        err = self.lib.openJPG(self.ptr, os.fsencode(path))
        if check and err:
            raise DecodeError(err, path)
        return err

    def open_bytes(self, data, check: bool = True) -> int:
        """Decode JPEG bytes (bytes, bytearray, uint8 ndarray, or a pinned
        torch tensor's data_ptr given as (ptr, size))."""
        if isinstance(data, tuple):
            ptr, size = data
        else:
            arr = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
            arr = np.ascontiguousarray(arr)
            self._pinned_src = arr  # keep alive during the call
            ptr, size = arr.ctypes.data, arr.nbytes
        err = self.lib.openJPGMem(self.ptr, C.c_void_p(ptr), size)
        if check and err:
            raise DecodeError(err)
        return err

    # ---- results
    def info(self) -> dict:
        a = (C.c_int64 * 12)()
        self.lib.cjReaderInfo(self.ptr, a)
        keys = ["width", "height", "channels", "mcux", "mcuy", "restart_interval", "bpm",
                "subsequences", "destuffed", "markers", "scan_bytes", "param_bytes"]
        return dict(zip(keys, [int(v) for v in a]))

    def pixels(self, copy: bool = True) -> np.ndarray:
        inf = self.info()
        h, w, ch = inf["height"], inf["width"], inf["channels"]
        n = w * h * (3 if ch == 3 else 1)
        p = self.lib.cjReaderPixels(self.ptr)
        if not p:
            raise DecodeError(PROGRAMMER_ERROR, "no decoded image")
        buf = (C.c_uint8 * n).from_address(p)
        arr = np.frombuffer(buf, np.uint8).reshape((h, w, 3) if ch == 3 else (h, w))
        return arr.copy() if copy else arr

    def stage_times(self) -> tuple:
        a = (C.c_float * 2)()
        self.lib.cjReaderStageTimes(self.ptr, a)
        return float(a[0]), float(a[1])

    def coefficients(self) -> list:
        """int32 dequantised coefficients per channel, [nblocks, 64] natural
        order, the reference's working_space layout.  Needs
        host_coefficients=True at construction."""
        out = []
        hdr = _reader_fields(self.ptr)
        for c in range(hdr["channels"]):
            mem, size = _working_space(self.ptr, c)
            if not mem:
                raise DecodeError(PROGRAMMER_ERROR, "coefficients were not exported")
            buf = (C.c_int32 * size).from_address(mem)
            out.append(np.frombuffer(buf, np.int32).copy().reshape(-1, 64))
        return out

    # ---- device-resident decode and instrumentation (benchmarks)
    def redecode_device(self):
        err = self.lib.cjReaderRedecodeDevice(self.ptr)
        if err:
            raise DecodeError(err, "redecode")

    def sync(self) -> int:
        return self.lib.cjReaderSync(self.ptr)

    def stream(self) -> int:
        return self.lib.cjReaderStream(self.ptr)

    def set_profile(self, on: bool):
        self.lib.cjReaderSetProfile(self.ptr, 1 if on else 0)

    def kernel_times(self) -> list:
        ids = (C.c_int * 32)()
        ms = (C.c_float * 32)()
        n = self.lib.cjReaderKernelTimes(self.ptr, ids, ms, 32)
        return [(KERNEL_NAMES[ids[k]], float(ms[k])) for k in range(n)]

    def launch_count(self) -> int:
        return int(self.lib.cjReaderLaunchCount(self.ptr))

    def plane_geometry(self, c: int) -> dict:
        """Arguments of cjIDCTPlane for component c of the last decode."""
        fields = _Reader.from_address(self.ptr)
        ch = fields.channels[c]
        first = sum(fields.channels[k].samples_x * fields.channels[k].samples_y for k in range(c))
        coef, _ = self.device_coefficients()
        return {"coef": coef, "bpm": self.info()["bpm"], "first": first, "sx": ch.samples_x,
                "sy": ch.samples_y, "mcux": fields.num_blocks_x, "mcuy": fields.num_blocks_y,
                "q": self.lib.cjReaderDeviceQuantTable(self.ptr, ch.dq_id), "rows": ch.block_stride,
                "stride": ch.stride}

    def plane_launch(self, geom: dict, out_ptr: int, mode: int, stream: int = 0):
        """Queue cjIDCTPlane for a plane_geometry() on `stream` (no sync)."""
        g = geom
        err = self.lib.cjIDCTPlane(C.c_void_p(g["coef"]), g["bpm"], g["first"], g["sx"], g["sy"],
                                   g["mcux"], g["mcuy"], C.c_void_p(g["q"]), C.c_void_p(out_ptr),
                                   g["stride"], mode, C.c_void_p(stream) if stream else None)
        if err:
            raise DecodeError(err, "cjIDCTPlane")

    def plane(self, c: int, mode: int = 0):
        """iDCT of component c of the last decode through cjIDCTPlane into a
        padded uint8 plane [rows, stride] (mode: IDCT_INT / IDCT_F32 / IDCT_TC)."""
        import torch
        g = self.plane_geometry(c)
        plane = torch.zeros((g["rows"], g["stride"]), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        self.plane_launch(g, plane.data_ptr(), mode)
        torch.cuda.synchronize()
        return plane.cpu().numpy()

    def device_coefficients(self):
        n = C.c_int64(0)
        p = self.lib.cjReaderDeviceCoefficients(self.ptr, C.byref(n))
        return p, n.value


class Batch:
    """The batched decoder (cudajpeg.h cjBatch*): one persistent kernel per
    batch of JPEGs of any size / subsampling / restart structure."""

    STAT_KEYS = ["submitted", "on_device", "grid", "warp_items", "destuff_tiles", "pixel_tiles",
                 "passes", "input_bytes", "output_bytes", "smem", "launches", "pixel_grid",
                 "graph_runs", "graph_failures", "blocks", "scan_bytes"]

    def __init__(self, sub_bits: int = 0):
        self.lib = load()
        self.ptr = self.lib.cjBatchCreate()
        if not self.ptr:
            raise MemoryError("cjBatchCreate failed")
        if sub_bits and self.lib.cjBatchSetSubsequenceBits(self.ptr, sub_bits):
            raise ValueError(f"bad subsequence size {sub_bits}")
        self.n = 0
        self._keep = None

    def close(self):
        if self.ptr:
            self.lib.cjBatchDestroy(self.ptr)
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

    @staticmethod
    def pack(files) -> tuple:
        """Concatenate JPEG byte strings -> (blob uint8 array, offsets, sizes)."""
        sizes = np.array([len(f) for f in files], np.int64)
        offsets = np.zeros(len(files), np.int64)
        if len(files):
            offsets[1:] = np.cumsum(sizes)[:-1]
        blob = np.frombuffer(b"".join(files), np.uint8) if files else np.zeros(1, np.uint8)
        return blob, offsets, sizes

    def stage(self, blob_ptr: int, offsets: np.ndarray, sizes: np.ndarray):
        offsets = np.ascontiguousarray(offsets, np.int64)
        sizes = np.ascontiguousarray(sizes, np.int64)
        self._keep = (offsets, sizes)
        self.n = len(sizes)
        err = self.lib.cjBatchStage(self.ptr, self.n, C.c_void_p(blob_ptr), offsets.ctypes.data,
                                    sizes.ctypes.data)
        if err:
            raise DecodeError(err, "cjBatchStage")

    def run(self):
        err = self.lib.cjBatchRun(self.ptr)
        if err:
            raise DecodeError(err, "cjBatchRun")

    def fetch(self):
        err = self.lib.cjBatchFetch(self.ptr)
        if err:
            raise DecodeError(err, "cjBatchFetch")

    def wait(self) -> list:
        errs = np.zeros(max(self.n, 1), np.int32)
        err = self.lib.cjBatchWait(self.ptr, errs.ctypes.data)
        if err:
            raise DecodeError(err, "cjBatchWait")
        return [int(e) for e in errs[: self.n]]

    def set_output(self, fmt: int = OUTPUT_RGB, idct: int = IDCT_INT):
        """Output format and pixel-stage iDCT of batches staged from now on."""
        if self.lib.cjBatchSetOutput(self.ptr, fmt, idct):
            raise ValueError(f"bad output {(fmt, idct)}")
        self.fmt = fmt

    def image(self, i: int, copy: bool = True):
        """Image i after a fetch: RGB [H, W, 3] / grey [H, W]; in the planar
        format a tuple (Y, Cb, Cr) of 2-D planes, in NV12 (Y, CbCr [ch, cw, 2])."""
        w, h, c = C.c_int(0), C.c_int(0), C.c_int(0)
        p = self.lib.cjBatchImage(self.ptr, i, C.byref(w), C.byref(h), C.byref(c))
        if not p:
            return None
        return _image_view(p, w.value, h.value, c.value, getattr(self, "fmt", OUTPUT_RGB),
                           self._chroma_size(i), copy)

    def device_tensor(self, i: int):
        """Image i of the last run as a torch tensor on the GPU, without a
        copy (cjBatchDLPack through the DLPack protocol).  A view of the
        batch's output buffer: valid until the batch is staged again or
        closed."""
        import torch
        p = self.lib.cjBatchDLPack(self.ptr, i)
        if not p:
            raise DecodeError(PROGRAMMER_ERROR, f"no device image {i}")
        return torch.from_dlpack(DLPackView(p, self.lib))

    def _chroma_size(self, i: int):
        """(cw, ch) of image i: the reference's channel sizes."""
        cw, ch = C.c_int(0), C.c_int(0)
        self.lib.cjBatchChromaGeometry(self.ptr, i, C.byref(cw), C.byref(ch))
        return cw.value, ch.value

    def decode(self, files) -> tuple:
        """Decode a list of JPEG byte strings -> (list of arrays or None, errors)."""
        blob, offsets, sizes = self.pack(files)
        self._blob = blob
        self.stage(blob.ctypes.data, offsets, sizes)
        self.run()
        self.fetch()
        errs = self.wait()
        return [self.image(i) if not e else None for i, e in enumerate(errs)], errs

    def coefficients(self, i: int, nblocks: int) -> np.ndarray:
        """Image i's quantised int16 blocks [n, 64] (natural order, MCU scan
        order, components interleaved) from the last run."""
        out = np.empty((nblocks, 64), np.int16)
        n = self.lib.cjBatchCopyCoefficients(self.ptr, i, out.ctypes.data, nblocks)
        if n < 0:
            raise DecodeError(int(n), "cjBatchCopyCoefficients")
        return out[:n]

    def stats(self) -> dict:
        a = (C.c_int64 * 16)()
        self.lib.cjBatchStats(self.ptr, a)
        return dict(zip(self.STAT_KEYS, [int(v) for v in a]))

    def kernel_ms(self) -> float:
        return float(self.lib.cjBatchKernelMs(self.ptr))

    def phase_ms(self) -> dict:
        a = (C.c_float * 16)()
        n = self.lib.cjBatchPhaseTimes(self.ptr, a)
        return {BATCH_PHASES[k]: float(a[k]) for k in range(n)}

    def stream(self) -> int:
        return self.lib.cjBatchStream(self.ptr)

    def set_tuning(self, sub_bits: int = 0, decode_ctas_per_sm: int = 0, pixel_tile_cap: int = 0):
        err = self.lib.cjBatchSetTuning(self.ptr, sub_bits, decode_ctas_per_sm, pixel_tile_cap)
        if err:
            raise ValueError(f"bad tuning {(sub_bits, decode_ctas_per_sm, pixel_tile_cap)}")

    def set_sub_bits_for(self, sampling_class: int, bits: int):
        """Subsequence size for one sampling class (SAMPLING_*; 0 = follow
        the batch-wide size), for batches staged from now on."""
        if self.lib.cjBatchSetSubsequenceBitsFor(self.ptr, sampling_class, bits):
            raise ValueError(f"bad subsequence size {bits} for class {sampling_class}")

    def set_parse(self, on_device: bool = True):
        """Parse the files' marker segments on the GPU (the default) or on the
        host, for batches staged from now on (cjBatchSetParse)."""
        if self.lib.cjBatchSetParse(self.ptr, 1 if on_device else 0):
            raise ValueError("cjBatchSetParse")

    def set_hypotheses(self, on: bool = True):
        """MCU-phase hypotheses in the entropy decode of latency-bound batches
        (cjBatchSetHypotheses; results identical either way)."""
        if self.lib.cjBatchSetHypotheses(self.ptr, 1 if on else 0):
            raise ValueError("cjBatchSetHypotheses")

    def set_wait_limit(self, polls: int):
        """Bound each grid-barrier wait of the decode kernel (0 = default)."""
        if self.lib.cjBatchSetWaitLimit(self.ptr, polls):
            raise ValueError("cjBatchSetWaitLimit")

    def wait_status(self) -> tuple:
        """(batch-level code, per-image codes) of the queued work, without
        raising: cjBatchWait's return value and its errors[]."""
        errs = np.zeros(max(self.n, 1), np.int32)
        err = self.lib.cjBatchWait(self.ptr, errs.ctypes.data)
        return int(err), [int(e) for e in errs[: self.n]]

    def tuning(self) -> dict:
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        self.lib.cjBatchGetTuning(self.ptr, C.byref(a), C.byref(b), C.byref(c))
        return {"sub_bits": a.value, "decode_ctas_per_sm": b.value, "pixel_tile_cap": c.value,
                "sub_bits_class": [self.lib.cjBatchGetSubsequenceBitsFor(self.ptr, k)
                                   for k in range(SAMPLING_CLASSES)]}

    def autotune(self, blob_ptr: int, offsets: np.ndarray, sizes: np.ndarray, reps: int = 3) -> dict:
        """Time the batch under every candidate tuning (cjBatchAutotune) and
        keep the fastest; the batch is left staged under it."""
        offsets = np.ascontiguousarray(offsets, np.int64)
        sizes = np.ascontiguousarray(sizes, np.int64)
        self._keep = (offsets, sizes)
        self.n = len(sizes)
        best = C.c_float(0.0)
        trials = (C.c_float * 64)()
        err = self.lib.cjBatchAutotune(self.ptr, self.n, C.c_void_p(blob_ptr), offsets.ctypes.data,
                                       sizes.ctypes.data, reps, C.byref(best), trials, 64)
        if err:
            raise DecodeError(err, "cjBatchAutotune")
        out = self.tuning()
        out["best_ms"] = round(best.value, 4)
        out["trials_ms"] = [round(trials[k], 4) for k in range(64) if trials[k] > 0]
        return out


# ---- JPGReader field access for the few fields ctypes needs (layout of
# include/format.h on LP64)
class _Managed(C.Structure):
    _fields_ = [("mem", C.c_void_p), ("size", C.c_uint), ("max_size", C.c_uint)]


class _Channel(C.Structure):
    _fields_ = [("id", C.c_int), ("dq_id", C.c_int), ("ac_id", C.c_int), ("dc_id", C.c_int),
                ("width", C.c_int), ("height", C.c_int), ("samples_x", C.c_int),
                ("samples_y", C.c_int), ("stride", C.c_int), ("block_stride", C.c_int),
                ("num_blocks", C.c_int), ("dc_cumulative_val", C.c_int),
                ("working_space", _Managed), ("pixels", _Managed)]


class _Reader(C.Structure):
    _fields_ = [("buf", C.c_void_p), ("pos", C.c_void_p), ("end", C.c_void_p),
                ("width", C.c_ushort), ("height", C.c_ushort),
                ("num_blocks_x", C.c_ushort), ("num_blocks_y", C.c_ushort),
                ("block_size_x", C.c_ushort), ("block_size_y", C.c_ushort),
                ("num_channels", C.c_ubyte), ("restart_interval", C.c_int),
                ("channels", _Channel * 3), ("pixels", C.c_void_p), ("max_pixels_size", C.c_int),
                ("dq_tables", (C.c_ubyte * 64) * 4), ("file_buf", _Managed),
                ("time", C.c_long), ("error", C.c_int), ("error_line", C.c_int),
                ("error_file", C.c_char_p), ("error_func", C.c_char_p),
                ("flags", C.c_int), ("scan_seen", C.c_int), ("huff_defined", C.c_int),
                ("dev", C.c_void_p)]


def _reader_fields(ptr) -> dict:
    r = _Reader.from_address(ptr)
    return {"channels": r.num_channels, "error": r.error, "time": r.time,
            "error_func": r.error_func}


def _working_space(ptr, c):
    r = _Reader.from_address(ptr)
    ws = r.channels[c].working_space
    return ws.mem, ws.size


def idct_blocks_raw(coef_q: np.ndarray, q_nat: np.ndarray, mode: int) -> np.ndarray:
    """Raw FP32 iDCT (before +128 / rounding / clip) of quantised int16 blocks
    [n, 64] sharing the natural-order quantisation table q_nat, on the GPU
    through cjIDCTBlocksRaw (mode IDCT_F32 or IDCT_TC)."""
    import torch
    lib = load()
    c = torch.from_numpy(np.ascontiguousarray(coef_q, np.int16).reshape(-1, 64)).cuda()
    q = torch.from_numpy(np.ascontiguousarray(q_nat, np.int16).reshape(64)).cuda()
    out = torch.empty((c.shape[0], 64), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    err = lib.cjIDCTBlocksRaw(C.c_void_p(c.data_ptr()), c.shape[0], C.c_void_p(q.data_ptr()),
                              C.c_void_p(out.data_ptr()), mode, None)
    if err:
        raise DecodeError(err, "cjIDCTBlocksRaw")
    torch.cuda.synchronize()
    return out.cpu().numpy()


_DESTRUCTOR = C.CFUNCTYPE(None, C.c_void_p)


@_DESTRUCTOR
def _capsule_destructor(capsule):
    """Frees a DLPack descriptor no consumer took (its capsule kept the name
    "dltensor"; a consumer renames it "used_dltensor" and owns it)."""
    api = C.pythonapi
    if api.PyCapsule_IsValid(C.c_void_p(capsule), b"dltensor"):
        p = api.PyCapsule_GetPointer(C.c_void_p(capsule), b"dltensor")
        load().cjDLPackFree(p)


class DLPackView:
    """One DLManagedTensor* from the library as a DLPack producer
    (``__dlpack__`` / ``__dlpack_device__``), for torch.from_dlpack and the
    like.  The decode work that writes the image is ordered on the library's
    stream; callers synchronise it (cjBatchWait) before consuming."""

    def __init__(self, ptr: int, lib):
        self.ptr = ptr
        self.lib = lib
        t = C.cast(C.c_void_p(ptr), C.POINTER(C.c_int32 * 4))  # data pointer, then DLDevice
        self.device_id = int(t.contents[3])

    def __dlpack_device__(self):
        return (2, self.device_id)  # kDLCUDA

    def __dlpack__(self, stream=None, **kwargs):
        if self.ptr is None:
            raise RuntimeError("DLPack tensor already exported")
        api = C.pythonapi
        api.PyCapsule_New.restype = C.py_object
        api.PyCapsule_New.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        api.PyCapsule_IsValid.argtypes = [C.c_void_p, C.c_char_p]
        api.PyCapsule_GetPointer.restype = C.c_void_p
        api.PyCapsule_GetPointer.argtypes = [C.c_void_p, C.c_char_p]
        cap = api.PyCapsule_New(self.ptr, b"dltensor", C.cast(_capsule_destructor, C.c_void_p))
        self.ptr = None
        return cap

    def __del__(self):
        if getattr(self, "ptr", None):
            self.lib.cjDLPackFree(self.ptr)
            self.ptr = None


def _image_view(p: int, w: int, h: int, c: int, fmt: int, chroma, copy: bool):
    if c != 3 or fmt not in (OUTPUT_PLANAR, OUTPUT_NV12):
        n = w * h * c
        arr = np.frombuffer((C.c_uint8 * n).from_address(p), np.uint8)
        arr = arr.reshape((h, w, 3) if c == 3 else (h, w))
        return arr.copy() if copy else arr
    cw, ch = chroma
    n = w * h + 2 * cw * ch
    flat = np.frombuffer((C.c_uint8 * n).from_address(p), np.uint8)
    flat = flat.copy() if copy else flat
    y = flat[: w * h].reshape(h, w)
    if fmt == OUTPUT_NV12:
        return y, flat[w * h:].reshape(ch, cw, 2)
    return y, flat[w * h: w * h + cw * ch].reshape(ch, cw), flat[w * h + cw * ch:].reshape(ch, cw)


def parse_compare(data: bytes) -> tuple:
    """(mismatch mask, host error, device-parse error) of cjDebugParseCompare:
    the batch decoder's marker parse (run on the host) against openJPGMem's
    marker loop on the same file.  Needs no GPU."""
    lib = load()
    # 64 KiB of zeros after the file: a malformed segment length must not let
    # a parser read beyond what it was given, and if one did, it stays in
    # this buffer
    buf = C.create_string_buffer(bytes(data) + bytes(65536), len(data) + 65536)
    e1, e2 = C.c_int(0), C.c_int(0)
    r = lib.cjDebugParseCompare(buf, len(data), C.byref(e1), C.byref(e2))
    return r, e1.value, e2.value


def build_info() -> dict:
    """cjBuildInfo: compute capabilities compiled into the library and the
    binary version of the device code the current GPU runs (0 without one)."""
    lib = load()
    archs = (C.c_int * 8)()
    ver = C.c_int(0)
    n = lib.cjBuildInfo(archs, 8, C.byref(ver))
    return {"archs": [int(archs[k]) for k in range(min(n, 8))], "binary_version": ver.value}


def idct_blocks_raw_device(coef_q, q_nat, mode: int):
    """cjIDCTBlocksRaw on device tensors: int16 blocks [n, 64] and the int16
    natural-order table [64] (both on the GPU) -> float32 [n, 64] on the GPU,
    queued on torch's current stream."""
    import torch
    lib = load()
    out = torch.empty((coef_q.shape[0], 64), dtype=torch.float32, device=coef_q.device)
    err = lib.cjIDCTBlocksRaw(C.c_void_p(coef_q.data_ptr()), coef_q.shape[0], C.c_void_p(q_nat.data_ptr()),
                              C.c_void_p(out.data_ptr()), mode,
                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if err:
        raise DecodeError(err, "cjIDCTBlocksRaw")
    return out


def decode(data, sub_bits: int = 0) -> np.ndarray:
    """Decode one JPEG (bytes) to an RGB / grey ndarray."""
    with Reader(sub_bits=sub_bits) as r:
        r.open_bytes(data)
        return r.pixels()
