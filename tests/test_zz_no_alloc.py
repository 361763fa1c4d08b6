"""cjDecodeNoAlloc: the decode entry point for callers that cannot allocate
device memory while decoding (its working memory is one static device array
held by the library).  Its output must equal openJPGMem's for the same file,
over two calls in a row that reuse the shared array.  Collected last so that
a run stopping at its first failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def no_alloc_decode(cj, data: bytes, out) -> tuple:
    lib = cj.load()
    w, h, c = C.c_int(0), C.c_int(0), C.c_int(0)
    err = lib.cjDecodeNoAlloc(data, len(data), C.c_void_p(out.data_ptr()), out.numel(), C.byref(w),
                              C.byref(h), C.byref(c), None)
    return err, w.value, h.value, c.value


def test_no_alloc_matches_openjpg_twice(cj):
    import torch

    files = [W.small_case(71, 640, 480, "420", 85, 0, "texture").data,
             W.small_case(72, 333, 200, "444", 92, 5, "noise").data]
    out = torch.zeros(640 * 480 * 3, dtype=torch.uint8, device="cuda")  # the caller's buffer
    for data in files:
        err, w, h, c = no_alloc_decode(cj, data, out)
        assert err == 0
        got = out[: w * h * c].cpu().numpy().reshape((h, w, 3) if c == 3 else (h, w))
        with cj.Reader() as r:
            r.open_bytes(data)
            want = r.pixels()
        assert np.array_equal(got, want)


def test_no_alloc_rejects_oversized_image(cj):
    import torch

    data = W.single_4096().data  # needs far more than the static working memory
    out = torch.empty(16, dtype=torch.uint8, device="cuda")
    err, w, h, c = no_alloc_decode(cj, data, out)
    assert (w, h, c) == (4096, 4096, 3)
    assert err in (cj.UNSUPPORTED_ERROR, cj.PROGRAMMER_ERROR)
    out = torch.empty(4096 * 4096 * 3, dtype=torch.uint8, device="cuda")
    err, *_ = no_alloc_decode(cj, data, out)
    assert err == cj.UNSUPPORTED_ERROR
