"""Multi-rank host logic of the decoder's one-process-per-GPU layout, run as
two gloo ranks on the CPU: the pixel-balanced partition of one batch, the
per-rank workload seeds, and the max/sum reductions the bench's whole-job
numbers are built from.  No GPU and no data-path collective are involved."""
import datetime
import os
import queue
import socket

import pytest

from conftest import ROOT

WEIGHTS = [((k * 7919) % 97 + 1) * (1 + (k % 5)) for k in range(41)]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from cudajpeg_b200 import replicas as R
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        r, local, w = R.rank_env()
        mine = R.partition(WEIGHTS, w)[r]
        load = float(sum(WEIGHTS[i] for i in mine))
        job = R.sum_over_ranks(load, dist)
        slowest = R.max_over_ranks(load, dist)
        marker = R.max_over_ranks(10.0 * r + 1.0, dist)
        dist.barrier()
        out.put((r, local, w, mine, load, job, slowest, marker, R.rank_seed(4, r)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = []
    try:
        for _ in range(world):
            res.append(out.get(timeout=120))
    except queue.Empty:
        pytest.fail("a rank did not report within 120 s")
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    res.sort()
    shares = [r[3] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(len(WEIGHTS)))   # a partition
    assert not set(shares[0]) & set(shares[1])
    loads = [r[4] for r in res]
    assert all(r[5] == sum(WEIGHTS) for r in res)                      # sum over ranks
    assert all(r[6] == max(loads) for r in res)                        # max over ranks
    assert all(r[7] == 11.0 for r in res)
    assert max(loads) - min(loads) <= max(WEIGHTS)                     # balanced
    assert [r[0] for r in res] == [0, 1] and all(r[2] == world for r in res)
    assert res[0][8] == 4 and res[1][8] == 5                           # per-rank seeds


def test_partition_single_rank_and_empty():
    from cudajpeg_b200 import replicas as R
    assert R.partition(WEIGHTS, 1) == [list(range(len(WEIGHTS)))]
    assert R.partition([], 3) == [[], [], []]
    parts = R.partition([5, 5, 5], 4)
    assert sorted(sum(parts, [])) == [0, 1, 2] and parts[3] == []
    assert R.max_over_ranks(3.5, None) == 3.5 and R.sum_over_ranks(2.0, None) == 2.0


def test_bench_workload_shards():
    """bench.py's per-rank workloads: --split partitions one batch, the
    default gives every rank its own batch (seed 4 + rank)."""
    import sys
    sys.path.insert(0, ROOT)
    import bench
    full = bench.Workload("mixed_batch", 8, 0, 1)
    parts = [bench.Workload("mixed_batch", 8, r, 2, split=True) for r in range(2)]
    assert sorted(parts[0].files + parts[1].files) == sorted(full.files)
    assert parts[0].pixels + parts[1].pixels == full.pixels
    weak1 = bench.Workload("mixed_batch", 8, 1, 2)
    assert len(weak1.files) == 8 and set(weak1.files).isdisjoint(full.files)


def test_bench_traffic_lookup():
    """The roofline's DRAM traffic comes from the committed ncu summaries of
    the default 1024-image batch; another batch size finds none."""
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.traffic_key("mixed_batch", 1024) == "mixed_batch"
    assert bench.traffic_key("mixed_batch", 128) == "mixed_batch_128"
    for k in ("k_decode_batch", "k_pixel_batch"):
        v = bench.read_traffic(k, bench.traffic_key("mixed_batch", 1024))
        assert v is not None and 1e8 < v < 1e10
        assert bench.read_traffic(k, bench.traffic_key("mixed_batch", 128)) is None
