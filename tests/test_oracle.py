"""The CPU oracle (oracle/jpeg_oracle.c) against the reference's own outputs:
the committed golden vectors (tests/golden/make_golden.py) and, where the
reference build oracle/_ref is present, freshly generated images."""
import numpy as np
import pytest

from cudajpeg_b200 import workloads as W


def test_oracle_matches_golden(golden, oracle_mod):
    assert len(golden) >= 30
    for name, case in golden.items():
        d = oracle_mod.decode(case["jpeg"].tobytes())
        assert d.error == int(case["error"]), name
        if d.error:
            continue
        ncoef = len([k for k in case if k.startswith("coef")])
        assert ncoef == d.nch, name
        for c in range(d.nch):
            assert np.array_equal(d.coefs[c], case[f"coef{c}"]), (name, c)
        if "pixels" in case:
            assert np.array_equal(d.pixels, case["pixels"]), name


@pytest.mark.parametrize("seed,w,h,mode,q,ri,content", [
    (31, 77, 45, "420", 83, 0, "texture"),
    (32, 120, 64, "422", 91, 4, "noise"),
    (33, 64, 64, "444", 67, 0, "smooth"),
    (34, 150, 20, "gray", 99, 3, "noise"),
])
def test_oracle_matches_reference_build(tmp_path, oracle_mod, seed, w, h, mode, q, ri, content):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built here")
    s = W.small_case(seed, w, h, mode, q, ri, content)
    p = tmp_path / "x.jpg"
    p.write_bytes(s.data)
    err, coefs = oracle_mod.ref_gpu_coefs(str(p))
    d = oracle_mod.decode(s.data)
    assert err == d.error == 0
    for a, b in zip(coefs, d.coefs):
        assert np.array_equal(a, b)
    px = oracle_mod.ref_cpu_pixels(str(p))
    if ri == 0:
        assert np.array_equal(px, d.pixels)
    else:
        assert px is None  # CPUonly rejects restart markers (decodeScanCPU.c:41-43)
    # every file, restart markers included, against the reference's own parts:
    # GPU-tree coefficients + CPUonly iDCT / upsampling / colour
    assert np.array_equal(oracle_mod.ref_cpu_pixels(str(p), restart=True), d.pixels)
    secs, px_count, fails = oracle_mod.ref_cpu_bench([str(p)], 2, 1)
    assert fails == 0 and px_count == 2 * w * h


def test_fp64_idct_within_one_of_integer(golden, oracle_mod):
    """The FP64 iDCT rounds to the reference's integer iDCT within +-1."""
    case = golden["c420_97x101_q100"]
    coef = case["coef0"]
    ref = oracle_mod.idct_int(coef).astype(np.int32)
    f = oracle_mod.idct_f64(coef)
    mine = np.clip(np.floor(f + 0.5) + 128, 0, 255).astype(np.int32)
    assert np.abs(mine - ref).max() <= 1
    assert (mine == ref).mean() > 0.9


def test_workloads_are_seeded():
    a = W.small_case(5, 40, 30, "420", 80, 2)
    b = W.small_case(5, 40, 30, "420", 80, 2)
    assert a.data == b.data
    batch = W.mixed_batch(n=24, seed=9, max_side=256)
    assert len(batch) == 24
    assert all(s.width % 8 == 0 and s.height % 8 == 0 for s in batch)


@pytest.mark.parametrize("mode,h,w", [("420", 64, 96), ("422", 48, 80), ("420", 40, 104), ("422", 24, 136)])
def test_fancy_upsampling_matches_libjpeg(oracle_mod, mode, h, w):
    """The oracle's fancy upsampler against Pillow's libjpeg decoding to
    YCbCr, on images whose blocks are all DC-only (content constant over
    each chroma block's footprint): there both decoders' iDCTs give
    round(DC / 8) + 128, so only the upsampling can differ."""
    import io

    from PIL import Image
    rng = np.random.default_rng(len(mode) + h + w)
    tile = (16, 16) if mode == "420" else (8, 16)
    t = rng.integers(30, 226, (h // tile[0], w // tile[1], 3)).astype(np.uint8)
    arr = np.kron(t, np.ones(tile + (1,), np.uint8))
    data = W.encode(arr, mode, 92)
    d = oracle_mod.decode(data, fancy=True)
    assert d.error == 0
    im = Image.open(io.BytesIO(data))
    im.draft("YCbCr", im.size)
    want = np.asarray(im)
    assert im.mode == "YCbCr" and want.shape == d.fancy_ycc.shape
    assert np.array_equal(d.fancy_ycc[..., 0], want[..., 0])  # luma: the DC-only iDCTs agree
    assert np.array_equal(d.fancy_ycc, want)
