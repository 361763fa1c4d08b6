"""The batched decoder (one persistent cooperative kernel per batch) against
the oracle: every image of a mixed batch -- uneven sizes, all subsampling
modes, restart intervals, corrupt files -- decodes exactly as alone."""
import numpy as np
import pytest

from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


def check_batch(cj, oracle_mod, files, sub_bits=0):
    with cj.Batch(sub_bits=sub_bits) as b:
        imgs, errs = b.decode(files)
        stats = b.stats()
    for k, data in enumerate(files):
        ref = oracle_mod.decode(data)
        assert errs[k] == ref.error, (k, errs[k], ref.error)
        if ref.error == 0:
            assert np.array_equal(imgs[k], ref.pixels), k
    return stats


def test_mixed_batch_matches_oracle(cj, oracle_mod):
    files = [s.data for s in W.mixed_batch(n=40, seed=21, max_side=700)]
    stats = check_batch(cj, oracle_mod, files)
    # staging: marker parse + header gather; the run: decode kernel + pixel kernel
    assert stats["on_device"] == 40 and stats["launches"] == 4
    assert stats["graph_runs"] == 1 and stats["graph_failures"] == 0  # launched as one CUDA graph


def test_golden_cases_in_one_batch(cj, golden, oracle_mod):
    """Valid, unsupported and corrupt files side by side: each keeps its own
    result (a corrupt file fails alone)."""
    names = sorted(golden)
    files = [golden[n]["jpeg"].tobytes() for n in names]
    with cj.Batch() as b:
        imgs, errs = b.decode(files)
    for n, img, e in zip(names, imgs, errs):
        case = golden[n]
        assert e == int(case["error"]), (n, e)
        if e == 0:
            ref = case["pixels"] if "pixels" in case else oracle_mod.decode(case["jpeg"].tobytes()).pixels
            assert np.array_equal(img, ref), n


@pytest.mark.parametrize("sub_bits", [256, 1024, 4096])
def test_batch_subsequence_sizes(cj, oracle_mod, sub_bits):
    files = [s.data for s in W.mixed_batch(n=12, seed=5, max_side=900)]
    check_batch(cj, oracle_mod, files, sub_bits)


def test_batch_rerun_and_large_image(cj, oracle_mod):
    big = W.single_4096().data
    files = [big] + [s.data for s in W.mixed_batch(n=6, seed=8, max_side=300)]
    with cj.Batch() as b:
        imgs, errs = b.decode(files)
        assert errs == [0] * len(files)
        first = [im.copy() for im in imgs]
        b.run()         # device-resident re-decode of the staged batch
        b.fetch()
        assert b.wait() == [0] * len(files)
        for k in range(len(files)):
            assert np.array_equal(b.image(k), first[k])
    assert np.array_equal(first[0], oracle_mod.decode(big).pixels)


def test_batch_same_result_alone_and_in_mix(cj):
    files = [s.data for s in W.mixed_batch(n=16, seed=33, max_side=600)]
    with cj.Batch() as b:
        mixed, errs = b.decode(files)
        assert all(e == 0 for e in errs)
        for k in (0, 5, 15):
            alone, e2 = b.decode([files[k]])
            assert e2 == [0] and np.array_equal(alone[0], mixed[k])


def test_batch_all_rejected_on_host(cj):
    with cj.Batch() as b:
        imgs, errs = b.decode([b"\xff\xd8\xff\xd9", b"not a jpeg at all"])
    assert errs == [1, 5] and imgs == [None, None]


@pytest.mark.parametrize("sub_bits,ctas,cap", [(512, 3, 0), (1024, 4, 0), (2048, 5, 4), (4096, 4, 2),
                                               (1024, 5, 8)])
def test_tuning_variants_identical(cj, oracle_mod, sub_bits, ctas, cap):
    """Every tuning the autotuner can pick decodes bit-identically."""
    files = [s.data for s in W.mixed_batch(n=16, seed=12, max_side=800)]
    with cj.Batch() as b:
        b.set_tuning(sub_bits, ctas, cap)
        imgs, errs = b.decode(files)
        t = b.tuning()
        assert (t["sub_bits"], t["decode_ctas_per_sm"], t["pixel_tile_cap"]) == (sub_bits, ctas, cap)
        assert t["sub_bits_class"] == [sub_bits] * cj.SAMPLING_CLASSES
    for k, data in enumerate(files):
        ref = oracle_mod.decode(data)
        assert errs[k] == ref.error, k
        if ref.error == 0:
            assert np.array_equal(imgs[k], ref.pixels), k


def test_per_class_subsequence_sizes(cj, oracle_mod):
    """A different subsequence size per sampling class in one batch (4:2:0
    long, grey short, 4:4:4 and 4:2:2 in between): results unchanged."""
    files = [s.data for s in W.mixed_batch(n=24, seed=14, max_side=900)]
    with cj.Batch() as b:
        for cls, bits in ((cj.SAMPLING_420, 16384), (cj.SAMPLING_GRAY, 256), (cj.SAMPLING_444, 8192),
                          (cj.SAMPLING_422, 1024)):
            b.set_sub_bits_for(cls, bits)
        with pytest.raises(ValueError):
            b.set_sub_bits_for(cj.SAMPLING_420, 100)
        assert b.tuning()["sub_bits_class"] == [16384, 1024, 8192, 256, 4096]
        imgs, errs = b.decode(files)
        b.set_sub_bits_for(cj.SAMPLING_420, 0)
        assert b.tuning()["sub_bits_class"][cj.SAMPLING_420] == 4096
    for k, data in enumerate(files):
        ref = oracle_mod.decode(data)
        assert errs[k] == ref.error, k
        if ref.error == 0:
            assert np.array_equal(imgs[k], ref.pixels), k


def test_autotune_keeps_results(cj, oracle_mod):
    files = [s.data for s in W.mixed_batch(n=24, seed=13, max_side=600)]
    blob, offsets, sizes = cj.Batch.pack(files)
    with cj.Batch() as b:
        res = b.autotune(blob.ctypes.data, offsets, sizes, reps=1)
        assert res["sub_bits"] in (512, 1024, 2048, 4096)
        assert all(x in (512, 1024, 2048, 4096, 8192, 16384) for x in res["sub_bits_class"])
        assert res["decode_ctas_per_sm"] in (3, 4, 5)
        assert res["best_ms"] > 0 and min(t for t in res["trials_ms"] if t > 0) == pytest.approx(res["best_ms"])
        b.run()
        b.fetch()
        errs = b.wait()
        for k, data in enumerate(files):
            ref = oracle_mod.decode(data)
            assert errs[k] == ref.error
            if ref.error == 0:
                assert np.array_equal(b.image(k), ref.pixels), k




def test_barrier_timeout_stops_the_batch(cj, oracle_mod):
    """A grid-barrier wait that runs out (a limit of one poll: the first CTAs
    at a barrier give up before the last arrive) ends the run with
    CUDA_KERNEL_LAUNCH_ERROR promptly, without running later phases on
    unsettled data; the same decoder then decodes the batch exactly."""
    import time

    files = [s.data for s in W.mixed_batch(n=24, seed=41, max_side=900)]
    blob, offsets, sizes = cj.Batch.pack(files)
    with cj.Batch() as b:
        b.stage(blob.ctypes.data, offsets, sizes)
        b.set_wait_limit(1)
        t0 = time.perf_counter()
        b.run()
        err, errs = b.wait_status()
        assert time.perf_counter() - t0 < 5.0
        assert err == cj.CUDA_KERNEL_LAUNCH_ERROR
        assert set(errs) == {cj.CUDA_KERNEL_LAUNCH_ERROR}
        b.set_wait_limit(0)
        b.run()
        b.fetch()
        errs = b.wait()
        for k, data in enumerate(files):
            ref = oracle_mod.decode(data)
            assert errs[k] == ref.error, k
            if ref.error == 0:
                assert np.array_equal(b.image(k), ref.pixels), k
