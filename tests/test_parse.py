"""The batch decoder's marker parse (cj_parse_header, which the GPU runs one
thread per file) against the drop-in path's host marker loop (openJPGMem up
to the scan: src/format.cu:159-215 and the segment checks of
src/format.cu:242-442, src/decodeScanGPU.cu:124-144): the same error code
for every file, and on success the same scan range and the same header byte
for byte.  Runs on the host (cjDebugParseCompare); no GPU needed.  Files:
the golden fixtures (12 malformed among them), seeded encodes of every
sampling mode, restart interval and progressive frames, and seeded
mutations of them (truncations, byte flips and segment-length changes in
the header)."""
import io

import numpy as np
import pytest
from PIL import Image

import cudajpeg_b200 as cj
from cudajpeg_b200 import workloads as W


def check(data: bytes, what):
    mask, e_host, e_parse = cj.parse_compare(data)
    assert mask == 0, (what, mask, e_host, e_parse)
    return e_host


def test_golden_files_parse_alike(golden):
    codes = set()
    for name in sorted(golden):
        data = np.asarray(golden[name]["jpeg"], np.uint8).tobytes()
        codes.add(check(data, name))
    assert 0 in codes and len(codes) > 2  # good files and several kinds of error


def encodes():
    out = []
    for k, (mode, w, h, q, ri) in enumerate([("420", 200, 136, 85, 0), ("422", 333, 200, 92, 4),
                                              ("444", 96, 80, 75, 0), ("gray", 150, 90, 90, 2),
                                              ("420", 17, 9, 60, 1), ("444", 1, 1, 50, 0)]):
        out.append(W.small_case(k + 70, w, h, mode, q, ri, "texture").data)
    rng = np.random.default_rng(5)
    img = Image.fromarray(rng.integers(0, 255, (64, 96, 3), dtype=np.uint8))
    for prog in (True, False):
        b = io.BytesIO()
        img.save(b, "JPEG", quality=80, progressive=prog, optimize=prog)
        out.append(b.getvalue())
    return out


def test_encodes_parse_alike():
    for k, data in enumerate(encodes()):
        check(data, k)


def test_mutations_parse_alike():
    rng = np.random.default_rng(11)
    n = 0
    for base in encodes():
        arr = np.frombuffer(base, np.uint8)
        # the header: up to the end of the first SOS segment
        sos = base.find(b"\xff\xda")
        hdr_end = sos + 2 + ((base[sos + 2] << 8) | base[sos + 3]) if sos > 0 else 64
        for cut in sorted(set(rng.integers(0, hdr_end + 8, 12).tolist())):
            check(base[:cut], ("cut", cut))                      # truncated, EOI lost
            check(base[:cut] + b"\xff\xd9", ("cut+eoi", cut))    # truncated, EOI kept
            n += 2
        for _ in range(60):
            m = arr.copy()
            for p in rng.integers(0, hdr_end, int(rng.integers(1, 4))):
                m[p] = rng.integers(0, 256) if rng.random() < 0.7 else m[p] ^ (1 << int(rng.integers(0, 8)))
            check(m.tobytes(), "flip")
            n += 1
        # segment lengths shortened / lengthened
        p = 2
        while p + 4 <= hdr_end and base[p] == 0xFF:
            ln = (base[p + 2] << 8) | base[p + 3]
            for d in (-3, -1, 1, 2, 300):
                m = bytearray(base)
                v = max(0, min(0xFFFF, ln + d))
                m[p + 2], m[p + 3] = v >> 8, v & 0xFF
                check(bytes(m), ("len", p, d))
                n += 1
            if base[p + 1] == 0xDA:
                break
            p += 2 + ln
    assert n > 500
