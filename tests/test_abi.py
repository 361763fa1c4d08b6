"""The C ABI of libcudajpeg.so without a GPU: every declared symbol is
exported, the header parser reproduces the reference's error codes, the
JPGReader layout seen through ctypes matches format.h, and the device
Huffman tables decode every 16-bit window like the reference's 64K table."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available


def declared_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(([^;{]*)\)\s*;", text, re.M):
            if m.group(1) not in ("if", "while", "return", "sizeof", "THROW"):
                names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(cj):
    names = declared_functions()
    assert {"openJPG", "decodeScanGPU", "iDCT_resample_colourTransform", "cjIDCTPlane"} <= names
    assert names == set(cj.EXPORTED)
    out = subprocess.run(["nm", "-D", "--defined-only", cj.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = names - syms
    assert not missing, missing


def test_library_has_sm100a_code(cj):
    """The library reports its device code as built for sm_100a only."""
    info = cj.build_info()
    assert info["archs"] == [1000], info
    if not gpu_available():
        assert info["binary_version"] == 0


HEADER_ONLY = ["bad_magic", "only_soi_eoi", "sof_precision_12", "sof2_progressive_marker",
               "dqt_16bit_id", "sos_component_count", "c420_3x9_unsupported"]


@pytest.mark.parametrize("name", HEADER_ONLY)
def test_header_errors_match_reference(cj, golden, name):
    """Errors raised before any device work: same code as the reference."""
    case = golden[name]
    with cj.Reader() as r:
        err = r.open_bytes(case["jpeg"].tobytes(), check=False)
    assert err == int(case["error"]), (name, err)


def test_reader_layout_and_geometry_without_gpu(cj, golden):
    if gpu_available():
        pytest.skip("checks the no-GPU path")
    case = golden["c420_130x66_opt"]
    with cj.Reader() as r:
        err = r.open_bytes(case["jpeg"].tobytes(), check=False)
        assert err == cj.CUDA_MEM_ERROR  # no CPU fallback: the scan needs a GPU
        info = r.info()
        assert (info["width"], info["height"], info["channels"]) == (130, 66, 3)
        assert (info["mcux"], info["mcuy"]) == (9, 5)
        fields = cj._Reader.from_address(r.ptr)
        assert fields.width == 130 and fields.height == 66 and fields.num_channels == 3
        assert fields.channels[1].samples_x == 1 and fields.channels[0].samples_x == 2
        assert fields.channels[0].stride == 9 * 16


def _reference_lut(counts, symbols):
    """The reference's 64K {num_bits, tuple} table (src/format.cu:372-391)."""
    lut = np.zeros(65536, np.int32)
    fill, k = 0, 0
    for l in range(1, 17):
        span = 1 << (16 - l)
        for _ in range(counts[l - 1]):
            lut[fill:fill + span] = (l << 8) | int(symbols[k])
            fill += span
            k += 1
    return lut


def _random_table(rng):
    # a random complete or incomplete prefix code with <= 256 symbols
    counts = [0] * 16
    left = 1 << 16
    nsym = 0
    for l in range(1, 17):
        cap = min(left >> (16 - l), 256 - nsym)
        n = int(rng.integers(0, cap + 1)) if l > 1 else int(rng.integers(0, 2))
        if l < 16:
            n = min(n, max(0, cap - 1))
        counts[l - 1] = n
        left -= n << (16 - l)
        nsym += n
    symbols = rng.integers(0, 256, nsym).astype(np.uint8)
    return counts, symbols


def test_huffman_tables_match_reference_lut(cj):
    lib = cj.load()
    rng = np.random.default_rng(0)
    annex_k_ac_luma = [0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7D]
    tables = [(annex_k_ac_luma, np.arange(162, dtype=np.uint8))]
    tables += [_random_table(rng) for _ in range(6)]
    for counts, symbols in tables:
        c = (C.c_ubyte * 16)(*counts)
        s = np.ascontiguousarray(symbols, np.uint8)
        ref = _reference_lut(counts, s)
        got = np.array([lib.cjDebugHuffDecode(c, s.ctypes.data, w) for w in range(0, 65536, 7)])
        assert np.array_equal(got, ref[::7])


def _step_of(e, ac):
    """Decode-step entry of a (len << 8 | symbol) table entry."""
    if not e:
        return 1 | (97 << 5)
    ln, sym = e >> 8, e & 255
    size, run = sym & 15, sym >> 4
    if not ac:
        dk = 1
    elif size:
        dk = run + 1
    else:
        dk = 64 if sym == 0 else (16 if sym == 0xF0 else 96)
    return (ln + size) | (dk << 5) | (size << 12)


def test_decode_steps_match_reference_lut(cj):
    """The two-level decode-step tables give, for every 16-bit window, the
    bits consumed / zig-zag advance / magnitude size of the reference's 64K
    table entry -- including tables with more long-code prefixes than
    subtables, which fall back to the canonical search."""
    lib = cj.load()
    rng = np.random.default_rng(1)
    annex_k_ac_luma = [0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7D]
    annex_k_dc_chroma = [0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0]
    many_long = [0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 120, 0, 0, 0, 0, 0]  # 120 codes of 11 bits: 60 prefixes
    tables = [(annex_k_ac_luma, np.arange(162, dtype=np.uint8), True),
              (annex_k_dc_chroma, np.arange(12, dtype=np.uint8), False),
              (many_long, rng.integers(0, 256, sum(many_long)).astype(np.uint8), True)]
    tables += [_random_table(rng) + (bool(k & 1),) for k in range(6)]
    vstep = np.vectorize(_step_of)
    for counts, symbols, ac in tables:
        c = (C.c_ubyte * 16)(*counts)
        s = np.ascontiguousarray(symbols, np.uint8)
        out = np.zeros(65536, np.uint16)
        assert lib.cjDebugStepTable(c, s.ctypes.data, int(ac), out.ctypes.data) == 0
        want = vstep(_reference_lut(counts, s), ac).astype(np.uint16)
        assert np.array_equal(out, want), (counts, ac, np.nonzero(out != want)[0][:5])


def test_batch_tuning_validation_without_gpu(cj):
    """cjBatchSetTuning checks its arguments on the host (no device work)."""
    with cj.Batch() as b:
        assert b.tuning() == {"sub_bits": 4096, "decode_ctas_per_sm": 4, "pixel_tile_cap": 0,
                              "sub_bits_class": [4096] * 5}
        b.set_tuning(2048, 5, 4)
        b.set_sub_bits_for(cj.SAMPLING_420, 8192)
        assert b.tuning() == {"sub_bits": 2048, "decode_ctas_per_sm": 5, "pixel_tile_cap": 4,
                              "sub_bits_class": [8192, 2048, 2048, 2048, 2048]}
        for bad in [(100, 4, 0), (1000, 4, 0), (1024, 7, 0), (1024, 2, 0), (1024, 4, 3), (1024, 4, -2)]:
            with pytest.raises(ValueError):
                b.set_tuning(*bad)
        for cls, bits in [(cj.SAMPLING_420, 96), (cj.SAMPLING_GRAY, 1000), (5, 1024), (-1, 1024)]:
            with pytest.raises(ValueError):
                b.set_sub_bits_for(cls, bits)
        assert b.tuning()["sub_bits"] == 2048  # a rejected call changes nothing
        assert b.tuning()["sub_bits_class"][cj.SAMPLING_420] == 8192
