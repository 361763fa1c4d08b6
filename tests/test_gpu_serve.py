"""The continuous-batching server (cudajpeg_b200.serve, cjServer*): every
request's result is the same alone and in a mix of concurrent requests, and
the same as the oracle; admission respects the device-bytes budget; the
open-loop replayer reports per-request latencies."""
import threading

import numpy as np
import pytest

from cudajpeg_b200 import serve as sv
from cudajpeg_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def samples():
    return W.mixed_batch(n=48, seed=31, max_side=640)


@pytest.fixture(scope="module")
def files(samples):
    return [s.data for s in samples]


def decode_alone(files):
    """Each file through its own server, one request at a time."""
    out = []
    with sv.Server(engines=1) as s:
        for f in files:
            t = s.submit(f)
            res = s.wait(t)
            out.append((res["error"], s.copy_out(t, res) if res["error"] == 0 else None))
            s.release(t)
        assert s.stats()["largest_batch"] == 1
    return out


def test_alone_and_in_mix_identical(cj, oracle_mod, files):
    alone = decode_alone(files)
    with sv.Server(engines=3) as s:
        tickets = [s.submit(f) for f in files]  # a burst: later requests join running ones
        mixed = []
        for t in tickets:
            res = s.wait(t)
            mixed.append((res["error"], s.copy_out(t, res) if res["error"] == 0 else None))
            s.release(t)
        st = s.stats()
    assert st["images"] == len(files)
    assert st["largest_batch"] > 1, st  # requests were batched together
    for k, f in enumerate(files):
        ref = oracle_mod.decode(f)
        assert alone[k][0] == mixed[k][0] == ref.error, k
        if ref.error == 0:
            assert np.array_equal(alone[k][1], mixed[k][1]), k
            assert np.array_equal(mixed[k][1], ref.pixels), k


def test_submitters_on_many_threads(cj, oracle_mod, files):
    results = {}
    with sv.Server(engines=2) as s:
        def client(idx):
            for k in idx:
                t = s.submit(files[k])
                res = s.wait(t)
                results[k] = s.copy_out(t, res)
                s.release(t)
        threads = [threading.Thread(target=client, args=(range(i, len(files), 4),)) for i in range(4)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
    for k, f in enumerate(files):
        assert np.array_equal(results[k], oracle_mod.decode(f).pixels), k


def test_budget_limits_batches(cj, oracle_mod, files):
    """A budget below one request's footprint: each request runs alone (a
    lone request is always admitted), results unchanged."""
    with sv.Server(engines=3, hbm_budget_bytes=1) as s:
        tickets = [s.submit(f) for f in files[:12]]
        for k, t in enumerate(tickets):
            res = s.wait(t)
            assert np.array_equal(s.copy_out(t, res), oracle_mod.decode(files[k]).pixels), k
            s.release(t)
        st = s.stats()
    assert st["largest_batch"] == 1 and st["batches"] == 12, st


def test_corrupt_request_fails_alone(cj, oracle_mod, files):
    bad = bytearray(files[0])
    bad[len(bad) // 2:] = b"\xff\xd9" + bytes(len(bad) - len(bad) // 2 - 2)
    mix = [files[1], bytes(bad), files[2], b"\x00\x01garbage", files[3]]
    with sv.Server(engines=2) as s:
        tickets = [s.submit(f) for f in mix]
        res = [s.wait(t) for t in tickets]
        for k, (f, r) in enumerate(zip(mix, res)):
            ref = oracle_mod.decode(f)
            assert r["error"] == ref.error, (k, r["error"], ref.error)
            if ref.error == 0:
                assert np.array_equal(s.copy_out(tickets[k], r), ref.pixels), k
        for t in tickets:
            s.release(t)


def test_replay_open_loop(cj, samples, files):
    arr = sv.poisson_arrivals(2000.0, 400, seed=1)
    px = np.array([s.pixels for s in samples], np.float64)
    with sv.Server(engines=3) as s:
        run = s.replay(files, arr)
        st = s.stats()
    summ = sv.summarize(run, px, 2000.0)
    assert summ["errors"] == 0
    assert (run["latency_ms"] > 0).all()
    assert st["images"] == 400 and st["waiting"] == 0
    assert summ["p50_ms"] <= summ["p99_ms"] <= summ["p999_ms"]
