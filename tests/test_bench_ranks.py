"""The bench's multi-rank timing on CPU: two gloo ranks, each with its own timed duration,
agree on the slowest one, and the whole-job throughput counts both ranks' work."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, durations, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(durations[rank], world, dist, "cpu")
        out.put((rank, ms, bench.aggregate_gbs(100_663_296, 10, world, ms)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_with_gloo():
    world, durations = 2, [12.5, 40.0]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, durations, out))
             for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [ms for _, ms, _ in results] == [40.0, 40.0]
    want = 100_663_296 * 10 * 2 / 0.040 / 1e9
    assert all(abs(v - want) < 1e-9 for _, _, v in results)


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.25, 1, None, "cpu") == 3.25
    assert bench.aggregate_gbs(1_000_000, 1000, 1, 1000.0) == 1.0
