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


def progressive_twins(mode, w, h, q, ri, seed):
    """The same pixels encoded baseline and progressive by Pillow's libjpeg:
    same quantisation, same coefficients, different scans."""
    import io

    from PIL import Image
    rng = np.random.default_rng(seed)
    arr = W.smooth_content(rng, w, h, 1 if mode == "gray" else 3)
    if mode == "gray":
        arr = arr[..., 0]
    out = []
    for prog in (False, True):
        buf = io.BytesIO()
        kw = dict(quality=q, optimize=False, progressive=prog)
        if mode != "gray":
            kw["subsampling"] = W.SUBSAMPLING[mode]
        if ri:
            kw["restart_marker_blocks"] = ri
        Image.fromarray(arr, "L" if mode == "gray" else "RGB").save(buf, "JPEG", **kw)
        out.append(buf.getvalue())
    return out


PROGRESSIVE_CASES = [("420", 200, 136, 85, 0), ("422", 333, 200, 92, 0), ("444", 96, 80, 75, 0),
                     ("gray", 150, 90, 90, 0), ("420", 257, 131, 60, 0), ("420", 128, 96, 80, 2),
                     ("444", 64, 64, 95, 3), ("420", 17, 9, 70, 0)]


@pytest.mark.parametrize("mode,w,h,q,ri", PROGRESSIVE_CASES)
def test_oracle_progressive_equals_baseline_twin(oracle_mod, mode, w, h, q, ri):
    """The oracle's progressive decode (T.81 Annex G) gives the coefficients
    and pixels of the baseline twin, which the reference decodes."""
    base, prog = progressive_twins(mode, w, h, q, ri, seed=w + h)
    assert prog.count(b"\xff\xda") > 1 and b"\xff\xc2" in prog
    a, b = oracle_mod.decode(base), oracle_mod.decode(prog)
    assert a.error == b.error == 0
    for x, y in zip(a.coefs, b.coefs):
        assert np.array_equal(x, y)
    assert np.array_equal(a.pixels, b.pixels)


def dqt_to_16bit(data: bytes, scale: int = 1) -> bytes:
    """Rewrite every 8-bit DQT table of a file as a 16-bit table (Pq = 1)
    holding the same values times `scale`."""
    out, i = bytearray(), 0
    while True:
        j = data.find(b"\xff\xdb", i)
        if j < 0 or j > data.find(b"\xff\xda"):
            out += data[i:]
            return bytes(out)
        n = (data[j + 2] << 8) | data[j + 3]
        seg, body = data[j + 4: j + 2 + n], bytearray()
        for k in range(0, len(seg), 65):
            body.append(0x10 | seg[k])
            for v in seg[k + 1: k + 65]:
                body += (v * scale).to_bytes(2, "big")
        out += data[i:j] + b"\xff\xdb" + (len(body) + 2).to_bytes(2, "big") + body
        i = j + 2 + n


def test_oracle_16bit_dqt(oracle_mod):
    s = W.small_case(51, 120, 88, "420", 80, 0, "texture")
    d8, d16 = oracle_mod.decode(s.data), oracle_mod.decode(dqt_to_16bit(s.data))
    assert d8.error == d16.error == 0 and np.array_equal(d8.pixels, d16.pixels)
    big = oracle_mod.decode(dqt_to_16bit(s.data, scale=12))  # steps above 255
    assert big.error == 0 and int(big.dq.max()) > 255
