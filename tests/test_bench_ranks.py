"""The bench's multi-GPU contract on CPU with two gloo ranks: timings are
the maximum over ranks, the whole-job rate sums the replicas' pairs, and the
reference arm does its work on rank 0 only (the other ranks exit 0 at once)."""
import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [10.0 + rank, 50.0 - rank]            # rank 1 is slower on the first timing
        got = bench.max_over_ranks(dist, ms)
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [11.0, 50.0]


def test_replica_rate_and_single_rank_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(None, [3.0, 4.0]) == [3.0, 4.0]
    # two replicas of 10 steps of 1e12 pairs in 2 s: 1e4 G interactions/s
    assert bench.replica_rate(2, 1e12, 10, 2000.0) == pytest.approx(1e4)


def test_reference_arm_is_rank_zero_only(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(bench.parse()) == 0   # no work, no output on rank 1


def test_force_flops_counts_each_kernel_form():
    """Executed FP32 flops per launch: 17 per ordered pair one-sided, 23 per
    unordered pair of different 1024-blocks for the pair kernel."""
    import bench
    assert bench.force_flops(1000, False) == 17.0 * 1000 * 1000
    own = 2.0 * 1024 * 1024
    assert bench.force_flops(2048, True) == 23.0 * (2048.0 ** 2 - own) / 2 + 17.0 * own
    own = 1024.0 ** 2 + 476.0 ** 2
    assert bench.force_flops(1500, True) == 23.0 * (1500.0 ** 2 - own) / 2 + 17.0 * own
    assert bench.force_flops(1024, True) == bench.force_flops(1024, False)
