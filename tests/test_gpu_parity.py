"""Parity of the CUDA decoder (through the C ABI) with the reference:
coefficients bit-exact with the reference's own decode, pixels bit-exact
with the reference CPUonly decoder (or the oracle restatement of it for
restart-marker files, which CPUonly cannot decode)."""
import ctypes

import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def decode_all(cj, data, sub_bits=0):
    with cj.Reader(sub_bits=sub_bits, host_coefficients=True) as r:
        err = r.open_bytes(data, check=False)
        if err:
            return err, None, None
        return 0, r.coefficients(), r.pixels()


def test_golden_cases(cj, golden, oracle_mod):
    for name, case in golden.items():
        data = case["jpeg"].tobytes()
        err, coefs, px = decode_all(cj, data)
        want = int(case["error"])
        assert err == want, (name, err, want)
        if err:
            continue
        for c, a in enumerate(coefs):
            assert np.array_equal(a, case[f"coef{c}"]), (name, c)
        ref_px = case["pixels"] if "pixels" in case else oracle_mod.decode(data).pixels
        assert np.array_equal(px, ref_px), name


@pytest.mark.parametrize("sub_bits", [128, 256, 512, 2048, 8192])
def test_subsequence_size_does_not_change_result(cj, golden, sub_bits):
    for name in ["c420_130x66_opt", "c422_200x120_ri5_opt", "c420_97x101_q100",
                 "gray_129x3_q95", "c420_160x96_ri7"]:
        case = golden[name]
        err, coefs, px = decode_all(cj, case["jpeg"].tobytes(), sub_bits)
        assert err == 0
        for c, a in enumerate(coefs):
            assert np.array_equal(a, case[f"coef{c}"]), (name, sub_bits)


CASES = [(100 + i, w, h, m, q, ri, cont) for i, (w, h, m, q, ri, cont) in enumerate([
    (640, 480, "420", 75, 0, "smooth"), (641, 479, "420", 95, 0, "noise"),
    (512, 512, "422", 88, 0, "texture"), (333, 257, "444", 92, 0, "noise"),
    (1000, 40, "gray", 97, 0, "noise"), (256, 256, "420", 70, 1, "texture"),
    (400, 300, "420", 85, 37, "noise"), (368, 200, "422", 60, 16, "smooth"),
    (200, 200, "444", 99, 5, "noise"), (800, 96, "gray", 80, 64, "texture"),
    (1920, 1080, "420", 90, 0, "texture"), (1023, 767, "444", 50, 0, "smooth"),
])]


@pytest.mark.parametrize("seed,w,h,mode,q,ri,content", CASES)
def test_random_images_against_oracle(cj, oracle_mod, seed, w, h, mode, q, ri, content):
    s = W.small_case(seed, w, h, mode, q, ri, content, optimize=(seed % 3 == 0 and content != "noise"))
    ref = oracle_mod.decode(s.data)
    assert ref.error == 0
    err, coefs, px = decode_all(cj, s.data)
    assert err == 0
    for c in range(ref.nch):
        assert np.array_equal(coefs[c], ref.coefs[c]), c
    assert np.array_equal(px, ref.pixels)


def test_reader_reuse_across_sizes(cj, oracle_mod):
    """One reader, grow-only buffers: large, small, colour, grey, restart."""
    samples = [W.small_case(7, 900, 700, "420", 90, 0, "texture"),
               W.small_case(8, 40, 24, "444", 75, 2, "noise"),
               W.small_case(9, 300, 200, "gray", 85, 0, "noise"),
               W.small_case(10, 1200, 100, "422", 65, 11, "smooth")]
    with cj.Reader() as r:
        for _ in range(2):
            for s in samples:
                r.open_bytes(s.data)
                assert np.array_equal(r.pixels(), oracle_mod.decode(s.data).pixels)


def test_single_1024_config(cj, oracle_mod):
    s = W.single_1024()
    ref = oracle_mod.decode(s.data)
    err, coefs, px = decode_all(cj, s.data)
    assert err == 0
    for c in range(3):
        assert np.array_equal(coefs[c], ref.coefs[c])
    assert np.array_equal(px, ref.pixels)


def test_single_4096_config(cj, oracle_mod):
    s = W.single_4096()
    ref = oracle_mod.decode(s.data)
    err, coefs, px = decode_all(cj, s.data)
    assert err == 0
    assert np.array_equal(px, ref.pixels)
    for c in range(3):
        assert np.array_equal(coefs[c], ref.coefs[c])


def test_restart_markers_do_not_change_coefficients_at_full_size(cj):
    """Size-independent property: the same pixels encoded with and without a
    restart interval carry identical coefficients, so decode identically."""
    rng = np.random.default_rng(11)
    arr = W.texture_content(rng, 4096, 2048, noise=5.0)
    plain = W.encode(arr, "420", 90, 0)
    rst = W.encode(arr, "420", 90, 17)
    with cj.Reader() as r:
        r.open_bytes(plain)
        a = r.pixels()
        r.open_bytes(rst)
        assert r.info()["markers"] > 100
        b = r.pixels()
    assert np.array_equal(a, b)


def test_entropy_corruption_agrees_with_reference(cj, golden):
    """Flipped bytes in the entropy data: the reference either rejects the
    file or decodes garbage; the GPU decoder does the same thing."""
    for name in ["flipped_byte_0", "flipped_byte_1", "flipped_byte_2", "truncated_scan",
                 "rst_wrong_index", "rst_missing"]:
        case = golden[name]
        err, coefs, px = decode_all(cj, case["jpeg"].tobytes())
        assert err == int(case["error"]), name
        if not err and "pixels" in case:
            assert np.array_equal(px, case["pixels"]), name


def test_reference_main_dropin(tmp_path, oracle_mod):
    """The reference's unmodified src/main.cu, built against include/ and
    libcudajpeg.so (oracle/_ref/main_dropin), decodes like the oracle."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(oracle_mod.__file__), "_ref", "main_dropin")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/main_dropin not built")
    for mode in ("420", "gray"):
        s = W.small_case(81, 301, 187, mode, 88, 0, "texture")
        p = tmp_path / f"in_{mode}.jpg"
        p.write_bytes(s.data)
        out = subprocess.run([exe, str(p)], cwd=tmp_path, capture_output=True, text=True, timeout=120)
        assert out.returncode == 0, out.stdout + out.stderr
        name = "outfile.pgm" if mode == "gray" else "outfile.ppm"
        raw = (tmp_path / name).read_bytes()
        header = b"P5\n301 187\n255\n" if mode == "gray" else b"P6\n301 187\n255\n"
        assert raw.startswith(header)
        px = np.frombuffer(raw[len(header):], np.uint8)
        assert np.array_equal(px, oracle_mod.decode(s.data).pixels.reshape(-1))


def test_device_code_runs_as_sm100(cj):
    """The device code the B200 runs is the library's own sm_100 binary (no
    PTX JIT of another target)."""
    assert cj.build_info()["binary_version"] == 100


def test_reference_alias_entry_points(cj, oracle_mod):
    """decodeScanCPU (include/decodeScanCPU.h:6) and the reference's
    alternative pixel stages (include/pixelTransformGPU.h:18-20) are GPU
    backed: a decode through the marker loop, then any of them, leaves the
    same image as the oracle's."""
    s = W.small_case(91, 300, 200, "420", 80, 0, "texture")
    ref = oracle_mod.decode(s.data)
    lib = cj.load()
    with cj.Reader() as r:
        r.open_bytes(s.data)
        for name in ("upsampleAndColourTransformGPU", "upsampleAndColourTransformHybrid",
                     "upsampleAndColourTransformCPU"):
            getattr(lib, name).argtypes = [ctypes.c_void_p]
            getattr(lib, name)(r.ptr)
            assert cj._reader_fields(r.ptr)["error"] == 0
            assert np.array_equal(r.pixels(), ref.pixels), name
    assert hasattr(lib, "decodeScanCPU")
