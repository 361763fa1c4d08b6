"""The batch decoder's other forms against the oracle.

* Planar and NV12 output: the decoded samples themselves (no upsampling, no
  colour transform), equal to the oracle's component planes cropped to the
  reference's channel sizes (src/format.cu:242-354 decodeSOF,
  src/pixelTransformGPU.cu:25-142 for the integer iDCT).
* The tensor-core iDCT (FP16 hi/lo basis, FP32 accumulation): every sample
  within +-1 of the integer iDCT's, with the exact fraction printed; every
  sample equal to the float64 iDCT rounded (clip(round(s) + 128)) except
  where s lies within 1e-3 of a rounding boundary, which bounds its error
  before rounding far below 0.5; RGB within the amplification of the colour
  transform.
"""
import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def component_planes(ref):
    """Oracle planes cropped to the channel sizes."""
    return [p[: c.height, : c.width] for p, c in zip(ref.planes, ref.comps)]


def f64_plane(oracle_mod, ref, c):
    """The float64 iDCT (before +128) of component c laid out as its plane."""
    comp = ref.comps[c]
    s = oracle_mod.idct_f64(ref.coefs[c])  # [n, 64], component scan order
    per = comp.samples_x * comp.samples_y
    j = np.arange(s.shape[0])
    mcu, loc = j // per, j % per
    bx = (mcu % ref.mcux) * comp.samples_x + loc % comp.samples_x
    by = (mcu // ref.mcux) * comp.samples_y + loc // comp.samples_x
    plane = np.zeros((comp.rows, comp.stride), np.float64)
    blocks = s.reshape(-1, 8, 8)
    for y in range(8):
        plane[(by * 8 + y)[:, None], bx[:, None] * 8 + np.arange(8)[None, :]] = blocks[:, y, :]
    return plane[: comp.height, : comp.width]


def decode_forms(cj, files, fmt, idct):
    with cj.Batch() as b:
        b.set_output(fmt, idct)
        imgs, errs = b.decode(files)
    return imgs, errs


FILES = [(81, 640, 480, "420", 85, 0, "texture"), (82, 333, 200, "444", 92, 5, "noise"),
         (83, 250, 190, "gray", 80, 0, "texture"), (84, 410, 302, "422", 60, 7, "texture"),
         (85, 129, 67, "420", 95, 0, "noise"), (86, 96, 1000, "444", 50, 0, "smooth")]


@pytest.fixture(scope="module")
def files():
    return [W.small_case(*a).data for a in FILES] + [s.data for s in W.mixed_batch(n=24, seed=44, max_side=900)]


def test_planar_and_nv12_equal_oracle_planes(cj, oracle_mod, files):
    planar, e1 = decode_forms(cj, files, cj.OUTPUT_PLANAR, cj.IDCT_INT)
    nv12, e2 = decode_forms(cj, files, cj.OUTPUT_NV12, cj.IDCT_INT)
    for k, data in enumerate(files):
        ref = oracle_mod.decode(data)
        assert e1[k] == e2[k] == ref.error, k
        if ref.error:
            continue
        want = component_planes(ref)
        if ref.nch == 1:
            assert np.array_equal(planar[k], want[0]) and np.array_equal(nv12[k], want[0]), k
            continue
        for c in range(3):
            assert np.array_equal(planar[k][c], want[c]), (k, c)
        assert np.array_equal(nv12[k][0], want[0]), k
        assert np.array_equal(nv12[k][1][..., 0], want[1]) and np.array_equal(nv12[k][1][..., 1], want[2]), k


def test_tensor_core_form(cj, oracle_mod, files):
    int_planes, e1 = decode_forms(cj, files, cj.OUTPUT_PLANAR, cj.IDCT_INT)
    tc_planes, e2 = decode_forms(cj, files, cj.OUTPUT_PLANAR, cj.IDCT_TC)
    int_rgb, e3 = decode_forms(cj, files, cj.OUTPUT_RGB, cj.IDCT_INT)
    tc_rgb, e4 = decode_forms(cj, files, cj.OUTPUT_RGB, cj.IDCT_TC)
    assert e1 == e2 == e3 == e4
    n = exact = 0
    rgb_n = rgb_within = rgb_max = 0
    for k, data in enumerate(files):
        if e1[k]:
            continue
        ref = oracle_mod.decode(data)
        a = int_planes[k] if ref.nch == 3 else (int_planes[k],)
        t = tc_planes[k] if ref.nch == 3 else (tc_planes[k],)
        for c in range(ref.nch):
            d = np.abs(a[c].astype(np.int16) - t[c].astype(np.int16))
            assert d.max() <= 1, (k, c)
            n += d.size
            exact += int((d == 0).sum())
            s = f64_plane(oracle_mod, ref, c)
            want = np.clip(np.floor(s + 0.5) + 128, 0, 255)
            miss = t[c] != want
            frac = np.abs(s - np.floor(s) - 0.5)
            # a mismatch with the rounded float64 iDCT only where the exact
            # value is within 1e-3 of .5: the error before rounding is < 1e-3
            assert not np.any(miss & (frac > 1e-3)), (k, c)
        rd = np.abs(int_rgb[k].astype(np.int16) - tc_rgb[k].astype(np.int16))
        rgb_n += rd.size
        rgb_within += int((rd <= 1).sum())
        rgb_max = max(rgb_max, int(rd.max()))
    print(f"tensor-core samples equal to the integer iDCT: {exact / n:.6f} of {n}; "
          f"RGB within +-1: {rgb_within / rgb_n:.6f}, max |diff| {rgb_max}")
    assert exact / n > 0.95
    assert rgb_max <= 3 and rgb_within / rgb_n > 0.99


def test_device_tensors_through_dlpack(cj, oracle_mod, files):
    """Decoded images handed to torch without a copy (cjBatchDLPack,
    cjServerDLPack): same bytes as the host copies and the oracle."""
    import torch

    from cudajpeg_b200 import serve as sv
    with cj.Batch() as b:
        imgs, errs = b.decode(files[:8])
        for k in range(8):
            t = b.device_tensor(k)
            assert t.is_cuda and t.dtype == torch.uint8 and tuple(t.shape) == imgs[k].shape
            assert t.data_ptr() == b.lib.cjBatchDeviceImage(b.ptr, k)  # a view, not a copy
            assert np.array_equal(t.cpu().numpy(), imgs[k])
            assert np.array_equal(imgs[k], oracle_mod.decode(files[k]).pixels)
        b.set_output(cj.OUTPUT_NV12, cj.IDCT_INT)
        imgs, errs = b.decode(files[:2])
        flat = b.device_tensor(0)
        y, cbcr = imgs[0]
        assert flat.dim() == 1 and flat.numel() == y.size + cbcr.size
        assert np.array_equal(flat.cpu().numpy(), np.concatenate([y.ravel(), cbcr.ravel()]))
    with sv.Server(engines=1) as s:
        tk = s.submit(files[0])
        res = s.wait(tk)
        t = s.device_tensor(tk)
        assert np.array_equal(t.cpu().numpy(), oracle_mod.decode(files[0]).pixels)
        del t
        s.release(tk)


def test_fancy_upsampling_equals_oracle(cj, oracle_mod, files):
    """CJ_OUTPUT_RGB_FANCY: the triangle-filter chroma upsampling (the
    oracle's restatement, pinned to libjpeg by tests/test_oracle.py) with the
    reference's iDCT and colour transform, bit-exact for every image; grey
    images are their plane."""
    rgb, errs = decode_forms(cj, files, cj.OUTPUT_RGB_FANCY, cj.IDCT_INT)
    fancy_differs = 0
    for k, data in enumerate(files):
        ref = oracle_mod.decode(data, fancy=True)
        assert errs[k] == ref.error, k
        if ref.error:
            continue
        want = ref.fancy_rgb if ref.nch == 3 else ref.pixels
        assert np.array_equal(rgb[k], want), k
        fancy_differs += int(not np.array_equal(want, ref.pixels))
    assert fancy_differs >= 10
