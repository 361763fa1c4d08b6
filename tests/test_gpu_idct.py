"""The three arithmetic forms of the plane iDCT (cjIDCTPlane):
integer (the reference's fixed point, bit-exact), FP32 CUDA cores, and FP16
hi/lo tensor cores (tcgen05) with FP32 accumulation -- the latter two within
0.5 of an FP64 iDCT before rounding, and within +-1 LSB of the reference."""
import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu

ZZ = np.array([0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48,
               41, 34, 27, 20, 13, 6, 7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15,
               23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63])


@pytest.mark.parametrize("mode,w,h", [("444", 512, 384), ("422", 512, 384), ("gray", 512, 384),
                                      ("420", 520, 392), ("420", 72, 40)])
def test_plane_forms(cj, oracle_mod, mode, w, h):
    s = W.small_case(61, w, h, mode, 95, 0, "noise")
    ref = oracle_mod.decode(s.data)
    with cj.Reader() as r:
        r.open_bytes(s.data)
        for c in range(ref.nch):
            pi = r.plane(c, cj.IDCT_INT)
            assert np.array_equal(pi, ref.planes[c]), c
            for form in (cj.IDCT_F32, cj.IDCT_TC):
                p = r.plane(c, form)
                diff = np.abs(p.astype(int) - ref.planes[c].astype(int))
                assert diff.max() <= 1, (c, form)
                assert (diff == 0).mean() > 0.95, (c, form)


def test_raw_error_against_fp64(cj, oracle_mod):
    s = W.small_case(62, 640, 480, "444", 95, 0, "noise")
    ref = oracle_mod.decode(s.data)
    q = np.zeros(64, np.int16)
    q[ZZ] = ref.dq[ref.comps[0].dq_id]
    quant = oracle_mod.quantised(ref)[0].astype(np.int16)
    exact = oracle_mod.idct_f64(ref.coefs[0])
    for form in (cj.IDCT_F32, cj.IDCT_TC):
        got = cj.idct_blocks_raw(quant, q, form)
        err = np.abs(got - exact)
        assert err.max() < 0.5 and err.mean() < 1e-3, (form, err.max(), err.mean())


def test_tensor_core_range_fallback(cj, oracle_mod):
    """Blocks whose dequantised values exceed FP16's exact range go to FP32."""
    rng = np.random.default_rng(3)
    quant = rng.integers(-20, 20, (300, 64)).astype(np.int16)
    quant[::7] = rng.integers(-20000, 20000, (43, 64))
    q = rng.integers(1, 100, 64).astype(np.int16)
    deq = quant.astype(np.int64) * q[None, :].astype(np.int64)
    exact = oracle_mod.idct_f64(deq.astype(np.int32))
    got = cj.idct_blocks_raw(quant, q, cj.IDCT_TC)
    # FP32 rounding error of a sum of 64 products scales with sum |F| / 8
    scale = np.maximum(1.0, np.abs(deq).sum(axis=1, keepdims=True) / 8.0)
    assert np.all(np.abs(got - exact) / scale < 1e-5)
    small = np.abs(deq).max(axis=1) <= 2048  # blocks that took the tensor-core path
    assert small.any() and (~small).any()
    assert np.abs(got[small] - exact[small]).max() < 0.5
