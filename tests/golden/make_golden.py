"""Generate tests/golden/golden.npz: small seeded JPEGs and the reference's
own outputs for them.

The reference (jndean/CUDAjpeg) ships no tests or golden vectors, so parity is
pinned on its executable code: oracle/Makefile builds
  oracle/_ref/libref_gputree.so  (src/format.cu + src/decodeScanCPU.cu) -> coefficients
  oracle/_ref/libref_cpuonly.so  (CPUonly decoder)                      -> pixels
from the reference sources, and this script records what they return.
CPUonly cannot decode restart-marker files (CPUonly/src/decodeScanCPU.c:41-43
re-inserts 0xFF instead of the RSTn byte), so for those only the coefficient
oracle's output and the error code are stored.

Run in a container that has the reference sources:
    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import io
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from cudajpeg_b200 import workloads as W  # noqa: E402

# (name, seed, w, h, mode, quality, restart, content, optimize)
CASES = [
    ("gray_16x16_q75", 1, 16, 16, "gray", 75, 0, "smooth", False),
    ("c420_33x17_q90", 2, 33, 17, "420", 90, 0, "noise", False),
    ("c422_40x24_q50", 3, 40, 24, "422", 50, 0, "smooth", False),
    ("c444_24x40_q95", 4, 24, 40, "444", 95, 0, "noise", False),
    ("c420_64x48_ri1", 5, 64, 48, "420", 80, 1, "smooth", False),
    ("c420_72x56_ri3", 6, 72, 56, "420", 70, 3, "noise", False),
    ("gray_50x30_ri2", 7, 50, 30, "gray", 60, 2, "noise", False),
    ("c444_8x8_q85", 8, 8, 8, "444", 85, 0, "smooth", False),
    ("c420_130x66_opt", 9, 130, 66, "420", 95, 0, "noise", True),
    ("gray_1x1", 10, 1, 1, "gray", 75, 0, "smooth", False),
    ("c444_1x1", 11, 1, 1, "444", 75, 0, "smooth", False),
    ("c420_3x9_unsupported", 12, 3, 9, "420", 75, 0, "smooth", False),
    ("c422_200x120_ri5_opt", 13, 200, 120, "422", 88, 5, "texture", True),
    ("c420_97x101_q100", 14, 97, 101, "420", 100, 0, "noise", False),
    ("c444_61x37_q1", 15, 61, 37, "444", 1, 0, "smooth", False),
    ("gray_129x3_q95", 16, 129, 3, "gray", 95, 0, "noise", False),
    ("c420_160x96_ri7", 17, 160, 96, "420", 85, 7, "texture", False),
    ("c422_48x48_ri9_final_full", 18, 48, 48, "422", 60, 9, "smooth", False),
    ("c444_40x40_ri100", 19, 40, 40, "444", 90, 100, "noise", False),
    ("c420_256x8_opt", 20, 256, 8, "420", 92, 0, "texture", True),
]


def malformed(cases: dict) -> dict:
    """Corrupted variants: byte edits that the reference rejects or accepts."""
    out = {}
    base = cases["c420_130x66_opt"]
    out["bad_magic"] = b"\x00" + base[1:]
    out["truncated_scan"] = base[: len(base) // 2] + b"\xff\xd9"
    sof = base.find(b"\xff\xc0")
    out["sof_precision_12"] = base[: sof + 4] + b"\x0c" + base[sof + 5:]
    out["sof2_progressive_marker"] = base[:sof] + b"\xff\xc2" + base[sof + 2:]
    dqt = base.find(b"\xff\xdb")
    out["dqt_16bit_id"] = base[: dqt + 4] + bytes([base[dqt + 4] | 0x10]) + base[dqt + 5:]
    sos = base.find(b"\xff\xda")
    out["sos_component_count"] = base[: sos + 4] + b"\x02" + base[sos + 5:]
    body = bytearray(base)
    rng = np.random.default_rng(7)
    for k in range(3):
        data = bytearray(base)
        lo = sos + 20
        idx = int(rng.integers(lo, len(data) - 4))
        data[idx] ^= 0x5A
        out[f"flipped_byte_{k}"] = bytes(data)
    rst = cases["c420_72x56_ri3"]
    p = rst.find(b"\xff\xd1")
    out["rst_wrong_index"] = rst[:p] + b"\xff\xd3" + rst[p + 2:]
    p = rst.find(b"\xff\xd0")
    out["rst_missing"] = rst[:p] + rst[p + 2:]
    out["only_soi_eoi"] = b"\xff\xd8\xff\xd9"
    del body
    return out


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref is not built (make -C oracle with the reference sources present)")
    jpegs = {}
    for name, seed, w, h, mode, q, ri, content, opt in CASES:
        jpegs[name] = W.small_case(seed, w, h, mode, q, ri, content, opt).data
    jpegs.update(malformed(jpegs))
    store = {}
    tmp = tempfile.mkdtemp()
    for name, data in jpegs.items():
        path = os.path.join(tmp, name + ".jpg")
        with open(path, "wb") as f:
            f.write(data)
        err, coefs = O.ref_gpu_coefs(path)
        px = O.ref_cpu_pixels(path)
        mine = O.decode(data)
        # the restatement must agree with the reference before it is trusted
        assert mine.error == err, (name, mine.error, err)
        for a, b in zip(coefs, mine.coefs):
            assert np.array_equal(a, b), name
        if px is not None:
            assert np.array_equal(px, mine.pixels), name
        store[f"{name}/jpeg"] = np.frombuffer(data, np.uint8)
        store[f"{name}/error"] = np.array(err, np.int32)
        for c, a in enumerate(coefs):
            store[f"{name}/coef{c}"] = a
        if px is not None:
            store[f"{name}/pixels"] = px
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **store)
    print(f"wrote {len(jpegs)} cases to {os.path.join(HERE, 'golden.npz')}")


if __name__ == "__main__":
    main()
