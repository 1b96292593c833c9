"""Replica bookkeeping of bench.py on CPU: two gloo ranks.

A single basin does not shard, so `bench.py --gpus N` runs N replicas and
reports the whole-job rate from the slowest rank's time.  These tests run the
same helpers bench.py uses over a world-size-2 gloo group.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, times, out):
    import torch.distributed as td
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    assert bench.dist() == (ws, rank, rank)
    td.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        t = bench.max_over_ranks(times[rank], td, "cpu")
        out.put((rank, t, bench.replica_value(t, ws, 1000, 10, 4)))
        td.barrier()
    finally:
        td.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [12.5, 20.0]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest rank's time
    assert [r[1] for r in res] == [20.0, 20.0]
    # 2 replicas x 1000 cells x 10 model steps x 4 steps in 20 ms
    assert res[0][2] == pytest.approx(2 * 1000 * 10 * 4 / 0.020 / 1e6)


def test_replica_value_single_rank():
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.replica_value(1000.0, 1, 513 * 513 * 3, 10, 5) == pytest.approx(
        513 * 513 * 3 * 50 / 1.0 / 1e6)


@pytest.mark.parametrize("ws", [1, 2, 3, 8])
def test_ensemble_shards_partition_the_members(ws):
    """N ranks step disjoint shards of the 256-member ensemble whose union is
    every member, each within one member of the others' counts; the
    whole-job rate counts the ensemble once (no replica factor)."""
    import bench
    shards = [bench.ensemble_shard(256, r, ws) for r in range(ws)]
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(256))
    assert max(map(len, shards)) - min(map(len, shards)) <= 1
    assert bench.replica_value(2000.0, 1, 10 ** 6, 10, 4) == pytest.approx(10 ** 6 * 40 / 2.0 / 1e6)
