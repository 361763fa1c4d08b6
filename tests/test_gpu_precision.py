"""The precision configuration at full size: 8192 x 8192 q95 images in 4:4:4,
4:2:2 and grey (50/50 uniform noise and gradient).  The plain path's pixels
equal the oracle's; per component, the integer plane iDCT equals the
oracle's plane, and the FP32 CUDA-core and FP16 hi/lo tensor-core forms
(cjIDCTPlane / cjIDCTBlocksRaw) stay within 0.5 of a float64 iDCT before
rounding and within +-1 LSB of the integer plane (the reference's iDCT,
src/pixelTransformGPU.cu:25-142), with the exact fraction printed."""
import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def idct_basis_f64():
    u = np.arange(8)[:, None]
    x = np.arange(8)[None, :]
    return np.where(u == 0, 1 / np.sqrt(2), 1.0) / 2 * np.cos((2 * x + 1) * u * np.pi / 16)


@pytest.mark.parametrize("mode", ["444", "422", "gray"])
def test_precision_8192(cj, oracle_mod, mode):
    import torch

    smp = W.precision_8192(mode)
    ref = oracle_mod.decode(smp.data)
    assert ref.error == 0
    basis = torch.from_numpy(idct_basis_f64()).cuda()
    ones = torch.ones(64, dtype=torch.int16, device="cuda")
    with cj.Reader(host_coefficients=True) as r:
        r.open_bytes(smp.data)
        assert np.array_equal(r.pixels(), ref.pixels)
        coefs = r.coefficients()
        for c in range(ref.nch):
            assert np.array_equal(coefs[c], ref.coefs[c]), c
            p_int = r.plane(c, cj.IDCT_INT)
            assert np.array_equal(p_int, ref.planes[c]), c
            dev = torch.from_numpy(coefs[c].astype(np.int16)).cuda()  # |dequantised| < 2^15 at q95
            for name, form in (("f32", cj.IDCT_F32), ("tc", cj.IDCT_TC)):
                plane = r.plane(c, form)
                diff = np.abs(plane.astype(np.int16) - p_int.astype(np.int16))
                exact = float((diff == 0).mean())
                print(f"{mode} component {c} {name}: exact {exact:.6f}, max |diff| {diff.max()}")
                assert diff.max() <= 1 and exact > 0.95, (c, name)
                worst = 0.0
                for k0 in range(0, dev.shape[0], 1 << 18):
                    blk = dev[k0:k0 + (1 << 18)].contiguous()
                    raw = cj.idct_blocks_raw_device(blk, ones, form)
                    x = blk.double().view(-1, 8, 8)
                    want = (basis.t() @ x @ basis).reshape(-1, 64)
                    worst = max(worst, float((raw.double() - want).abs().max()))
                torch.cuda.synchronize()
                print(f"{mode} component {c} {name}: max |error| vs float64 {worst:.3e}")
                assert worst < 0.5, (c, name, worst)
