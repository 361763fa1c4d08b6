"""cjDecodeNoAlloc: the decode entry point for callers that cannot allocate
device memory while decoding (its working memory is one static device array
held by the library).  Its output must equal openJPGMem's for the same file,
and the oracle's, over calls in a row that reuse the shared array.  Collected
last so that a run stopping at its first failure has run every other test
before it."""
import ctypes as C

import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def no_alloc_decode(cj, data: bytes, ptr: int, capacity: int) -> tuple:
    lib = cj.load()
    w, h, c = C.c_int(0), C.c_int(0), C.c_int(0)
    err = lib.cjDecodeNoAlloc(data, len(data), C.c_void_p(ptr), capacity, C.byref(w), C.byref(h),
                              C.byref(c), None)
    return err, w.value, h.value, c.value


def as_image(flat, w, h, c):
    return flat[: w * h * c].cpu().numpy().reshape((h, w, 3) if c == 3 else (h, w))


def open_jpg_mem(cj, data):
    with cj.Reader() as r:
        r.open_bytes(data)
        return r.pixels()


FILES = [(71, 640, 480, "420", 85, 0, "texture"), (72, 333, 200, "444", 92, 5, "noise"),
         (73, 250, 190, "gray", 80, 0, "texture"), (74, 410, 300, "422", 60, 7, "texture")]


def test_no_alloc_matches_openjpg_twice(cj, oracle_mod):
    """Two calls in a row for each file (4:2:0, 4:4:4 with restarts, grey,
    4:2:2 with restarts): each equals openJPGMem and the oracle."""
    import torch

    out = torch.zeros(640 * 480 * 3, dtype=torch.uint8, device="cuda")  # the caller's buffer
    for args in FILES:
        data = W.small_case(*args).data
        want = open_jpg_mem(cj, data)
        ref = oracle_mod.decode(data)
        assert ref.error == 0 and np.array_equal(want, ref.pixels)
        for _ in range(2):
            out.fill_(0x5A)
            err, w, h, c = no_alloc_decode(cj, data, out.data_ptr(), out.numel())
            assert err == 0 and (w, h) == (args[1], args[2])
            assert c == (1 if args[3] == "gray" else 3)
            assert np.array_equal(as_image(out, w, h, c), want)


def test_no_alloc_unaligned_output(cj):
    """An output pointer that is not 8-byte aligned (and an image width that is
    not a multiple of 8) takes the byte-store path of the pixel kernel."""
    import torch

    data = W.small_case(75, 203, 117, "420", 75, 0, "texture").data
    want = open_jpg_mem(cj, data)
    buf = torch.zeros(203 * 117 * 3 + 1, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        err, w, h, c = no_alloc_decode(cj, data, buf.data_ptr() + 1, buf.numel() - 1)
        assert err == 0
        assert np.array_equal(as_image(buf[1:], w, h, c), want)
    assert int(buf[0]) == 0  # nothing written before the caller's pointer


def test_no_alloc_small_output_buffer(cj):
    """An image that fits the static array but not the caller's buffer is
    refused before any GPU work: PROGRAMMER_ERROR, buffer untouched."""
    import torch

    data = W.small_case(76, 96, 64, "444", 90, 0, "noise").data
    need = 96 * 64 * 3
    buf = torch.full((need,), 0x33, dtype=torch.uint8, device="cuda")
    err, w, h, c = no_alloc_decode(cj, data, buf.data_ptr(), need - 1)
    assert err == cj.PROGRAMMER_ERROR and (w, h, c) == (96, 64, 3)
    torch.cuda.synchronize()
    assert bool((buf == 0x33).all())
    err, *_ = no_alloc_decode(cj, data, buf.data_ptr(), need)
    assert err == 0 and np.array_equal(as_image(buf, w, h, c), open_jpg_mem(cj, data))


def test_no_alloc_rejects_oversized_image(cj):
    import torch

    data = W.single_4096().data  # needs far more than the static working memory
    out = torch.empty(16, dtype=torch.uint8, device="cuda")
    err, w, h, c = no_alloc_decode(cj, data, out.data_ptr(), out.numel())
    assert (w, h, c) == (4096, 4096, 3)
    assert err in (cj.UNSUPPORTED_ERROR, cj.PROGRAMMER_ERROR)
    out = torch.empty(4096 * 4096 * 3, dtype=torch.uint8, device="cuda")
    err, *_ = no_alloc_decode(cj, data, out.data_ptr(), out.numel())
    assert err == cj.UNSUPPORTED_ERROR
