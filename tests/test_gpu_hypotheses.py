"""MCU-phase hypotheses in the entropy decode (latency-bound batches and the
drop-in path): the settle may continue from a decode that started under
another MCU phase, which changes only how long it takes.  The same batch
decoded with and without them gives identical coefficients and pixels, and
the single-image path (which uses them, with the probe decodes from each
predecessor hypothesis that settle a warp in one step) matches the oracle."""
import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_hypotheses_do_not_change_results(cj, oracle_mod):
    files = [s.data for s in W.mixed_batch(n=24, seed=91, max_side=1200)]
    files += [W.small_case(92, 640, 480, "420", 75, 0, "texture").data,
              W.small_case(93, 600, 400, "422", 90, 5, "noise").data,
              W.small_case(94, 512, 256, "444", 60, 0, "smooth").data]
    out = {}
    for on in (False, True):
        with cj.Batch() as b:
            b.set_hypotheses(on)
            imgs, errs = b.decode(files)
            out[on] = (imgs, errs)
    (i0, e0), (i1, e1) = out[False], out[True]
    assert e0 == e1
    for k in range(len(files)):
        if not e0[k]:
            assert np.array_equal(i0[k], i1[k]), k
    for k, data in enumerate(files):
        ref = oracle_mod.decode(data)
        assert e1[k] == ref.error, k
        if not ref.error:
            assert np.array_equal(i1[k], ref.pixels), k


# restart intervals put segment starts inside warps: a subsequence whose
# predecessor starts a segment has one predecessor hypothesis only
@pytest.mark.parametrize("case", [("420", 1024, 768, 75, 0), ("422", 900, 700, 85, 0), ("444", 640, 480, 95, 0),
                                  ("420", 1024, 768, 75, 3), ("420", 800, 600, 60, 17), ("422", 640, 480, 90, 40)])
def test_single_image_path_with_hypotheses(cj, oracle_mod, case):
    mode, w, h, q, restart = case
    s = W.small_case(95, w, h, mode, q, restart, "texture")
    ref = oracle_mod.decode(s.data)
    with cj.Reader(host_coefficients=True) as r:
        r.open_bytes(s.data)
        px = r.pixels()
        coefs = r.coefficients()
    assert np.array_equal(px, ref.pixels)
    for c in range(ref.nch):
        assert np.array_equal(coefs[c], ref.coefs[c]), c
