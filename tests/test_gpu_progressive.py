"""Progressive JPEG (SOF2) and 16-bit quantisation tables through the
drop-in path (openJPGMem), which the reference rejects (src/format.cu:191-200
and :432).  Pinned by twins: a progressive file and its baseline twin (the
same pixels encoded by the same libjpeg at the same quality, hence the same
quantised coefficients) must decode to the same coefficients and pixels, and
those of the baseline twin are the reference's; the oracle's progressive
decode (ITU T.81 Annex G) must agree as well."""
import numpy as np
import pytest

from test_oracle import PROGRESSIVE_CASES, dqt_to_16bit, progressive_twins

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,w,h,q,ri", PROGRESSIVE_CASES + [("420", 1024, 768, 75, 0), ("422", 640, 480, 90, 4)])
def test_progressive_equals_baseline_twin(cj, oracle_mod, mode, w, h, q, ri):
    base, prog = progressive_twins(mode, w, h, q, ri, seed=w + h)
    ref = oracle_mod.decode(base)
    assert ref.error == 0
    assert oracle_mod.decode(prog).error == 0
    for data in (prog, base):
        with cj.Reader(host_coefficients=True) as r:
            r.open_bytes(data)
            assert np.array_equal(r.pixels(), ref.pixels)
            for c, coef in enumerate(r.coefficients()):
                assert np.array_equal(coef, ref.coefs[c]), c


def test_progressive_then_baseline_on_one_reader(cj, oracle_mod):
    """A reader keeps working across frame types."""
    base, prog = progressive_twins("420", 300, 200, 80, 0, seed=9)
    other = W.small_case(12, 160, 120, "444", 85, 2, "texture").data
    with cj.Reader() as r:
        for data in (prog, other, prog, base):
            r.open_bytes(data)
            assert np.array_equal(r.pixels(), oracle_mod.decode(data).pixels)


def test_progressive_in_a_batch_is_unsupported(cj, oracle_mod):
    base, prog = progressive_twins("420", 120, 96, 85, 0, seed=3)
    with cj.Batch() as b:
        imgs, errs = b.decode([base, prog, base])
    assert errs == [0, cj.UNSUPPORTED_ERROR, 0]
    assert np.array_equal(imgs[2], oracle_mod.decode(base).pixels)


def test_16bit_quantisation_tables(cj, oracle_mod):
    s = W.small_case(52, 200, 136, "420", 85, 0, "texture")
    for data in (dqt_to_16bit(s.data), dqt_to_16bit(s.data, scale=12)):
        ref = oracle_mod.decode(data)
        assert ref.error == 0
        with cj.Reader() as r:
            r.open_bytes(data)
            assert np.array_equal(r.pixels(), ref.pixels)
        with cj.Batch() as b:  # the batch decoder reads 16-bit tables too
            imgs, errs = b.decode([data])
            assert errs == [0] and np.array_equal(imgs[0], ref.pixels)
    assert np.array_equal(oracle_mod.decode(dqt_to_16bit(s.data)).pixels, oracle_mod.decode(s.data).pixels)


def test_corrupt_progressive_scans_fail(cj, oracle_mod):
    """Corrupt progressive files fail (or decode) exactly as the oracle."""
    _, prog = progressive_twins("420", 160, 120, 85, 0, seed=4)
    rng = np.random.default_rng(11)
    sos = prog.find(b"\xff\xda")
    for k in range(12):
        data = bytearray(prog)
        idx = int(rng.integers(sos + 16, len(data) - 4))
        data[idx] ^= 0x5A
        data = bytes(data)
        ref = oracle_mod.decode(data)
        with cj.Reader() as r:
            err = r.open_bytes(data, check=False)
            if ref.error == 0 and err == 0:
                assert np.array_equal(r.pixels(), ref.pixels), k
            else:
                assert err != 0 and ref.error != 0, (k, err, ref.error)
