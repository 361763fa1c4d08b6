"""The benchmark's own workloads against the oracle, at full size.

* The mixed 1024-image batch (sides log-uniform in [64, 2048], 4:2:0 / 4:2:2 /
  4:4:4 / grey, q 50-95, 30% with restart intervals; seed 4) decoded in ONE
  cjBatch run: every image's error code and pixels equal the oracle's, and
  its quantised coefficients equal the oracle's dequantised coefficients
  divided by the quantisation table (src/decodeScanGPU.cu:435-490 for the
  coefficients, CPUonly/src/pixelTransformCPU.c:110-172 for the pixels).
* The same 1024 files as single-image requests to the continuous-batching
  server, submitted from two threads at once: each result equals the oracle.
"""
import os
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from cudajpeg_b200 import serve as sv
from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu

ZZ = np.array([0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48,
               41, 34, 27, 20, 13, 6, 7, 14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15,
               23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63])


@pytest.fixture(scope="module")
def headline():
    workers = max(1, min(32, os.cpu_count() or 1))
    return W.mixed_batch(n=1024, seed=4, workers=workers)


def oracle_pool():
    return ThreadPoolExecutor(max(1, min(32, os.cpu_count() or 1)))


def split_components(quant_blocks: np.ndarray, ref) -> list:
    """Batch blocks (MCU order, components interleaved) -> per-component
    dequantised int32 [n, 64] in the reference's working_space order."""
    sizes = [c.samples_x * c.samples_y for c in ref.comps]
    bpm = sum(sizes)
    mcus = quant_blocks.shape[0] // bpm
    per_mcu = quant_blocks.reshape(mcus, bpm, 64).astype(np.int32)
    out, first = [], 0
    for comp, n in zip(ref.comps, sizes):
        q = np.zeros(64, np.int32)
        q[ZZ] = ref.dq[comp.dq_id]
        out.append((per_mcu[:, first:first + n, :] * q).reshape(-1, 64))
        first += n
    return out


def test_headline_batch_matches_oracle(cj, oracle_mod, headline):
    files = [s.data for s in headline]
    with cj.Batch() as b:
        imgs, errs = b.decode(files)
        assert b.stats()["on_device"] == len(files)
        with oracle_pool() as ex:
            refs = ex.map(oracle_mod.decode, files)
            checked = restart = 0
            for k, ref in enumerate(refs):
                s = headline[k]
                assert errs[k] == ref.error, (k, errs[k], ref.error)
                if ref.error:
                    continue
                assert np.array_equal(imgs[k], ref.pixels), (k, s.width, s.height, s.mode, s.restart)
                nblocks = sum(c.nblocks for c in ref.comps)
                got = split_components(b.coefficients(k, nblocks), ref)
                for c in range(ref.nch):
                    assert np.array_equal(got[c], ref.coefs[c]), (k, c)
                checked += 1
                restart += s.restart > 0
    assert checked == len(files) and restart > 200, (checked, restart)


def test_headline_files_through_the_server(cj, oracle_mod, headline):
    """Config-4-sized requests, from two submitting threads, overlap on the
    GPU in continuous batches; every result equals the oracle."""
    import time

    files = [s.data for s in headline]
    tickets = {}
    with sv.Server(engines=3, hbm_budget_bytes=4 << 30) as s:
        def submit(part):
            for k in part:
                tickets[k] = s.submit(files[k])
        threads = [threading.Thread(target=submit, args=(range(j, len(files), 2),)) for j in (0, 1)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        # collect results as they finish (any order) and release them at once,
        # so finished engines are reused while later requests still wait
        got, pending = {}, set(tickets)
        deadline = time.monotonic() + 300
        while pending and time.monotonic() < deadline:
            before = len(pending)
            for k in list(pending):
                try:
                    res = s.wait(tickets[k], timeout_s=0.0)
                except TimeoutError:
                    continue
                got[k] = (res["error"], s.copy_out(tickets[k], res) if res["error"] == 0 else None)
                s.release(tickets[k])
                pending.discard(k)
            if len(pending) == before:
                time.sleep(0.002)
        assert not pending, f"{len(pending)} requests unfinished"
        st = s.stats()
    assert st["images"] == len(files) and st["largest_batch"] > 1, st
    with oracle_pool() as ex:
        for k, ref in enumerate(ex.map(oracle_mod.decode, files)):
            assert got[k][0] == ref.error, k
            if ref.error == 0:
                assert np.array_equal(got[k][1], ref.pixels), k


def test_headline_batch_tensor_core_form(cj, headline):
    """The batched tensor-core iDCT over the whole headline batch: every
    decoded sample (planar output) within +-1 of the integer iDCT's, the
    exact fraction printed; RGB within the colour transform's amplification."""
    files = [s.data for s in headline]
    out = {}
    for fmt, idct in ((cj.OUTPUT_PLANAR, cj.IDCT_INT), (cj.OUTPUT_PLANAR, cj.IDCT_TC), (cj.OUTPUT_RGB, cj.IDCT_TC)):
        with cj.Batch() as b:
            b.set_output(fmt, idct)
            imgs, errs = b.decode(files)
            assert not any(errs)
            out[(fmt, idct)] = imgs
    with cj.Batch() as b:
        rgb_int, errs = b.decode(files)
    n = exact = rgb_n = rgb_within = rgb_max = 0
    for k, s in enumerate(headline):
        a, t = out[(cj.OUTPUT_PLANAR, cj.IDCT_INT)][k], out[(cj.OUTPUT_PLANAR, cj.IDCT_TC)][k]
        planes = zip(a, t) if s.mode != "gray" else [(a, t)]
        for pa, pt in planes:
            d = np.abs(pa.astype(np.int16) - pt.astype(np.int16))
            assert d.max() <= 1, k
            n += d.size
            exact += int((d == 0).sum())
        rd = np.abs(rgb_int[k].astype(np.int16) - out[(cj.OUTPUT_RGB, cj.IDCT_TC)][k].astype(np.int16))
        rgb_n += rd.size
        rgb_within += int((rd <= 1).sum())
        rgb_max = max(rgb_max, int(rd.max()))
    print(f"headline batch, tensor-core iDCT: samples equal to the integer iDCT {exact / n:.6f} of {n}; "
          f"RGB within +-1 {rgb_within / rgb_n:.6f}, max |diff| {rgb_max}")
    assert exact / n > 0.95 and rgb_max <= 3 and rgb_within / rgb_n > 0.99
