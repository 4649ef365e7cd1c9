"""CPU: the multi-rank plumbing of bench.py (one process per GPU; replicas,
barrier and the max over ranks) on two gloo ranks, and the reference arm's
rank gating (rank 0 alone works)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    r = bench.Ranks("gloo", timeout_s=60)
    r.barrier()
    # each replica "took" a different time; the job is as slow as its slowest rank
    ms = 100.0 + 25.0 * rank
    got = r.max_over_ranks(ms)
    q.put((rank, r.world, got, bench.replica_throughput(r.world, 10, got)))
    r.barrier()
    r.close()


def test_two_gloo_ranks_max_and_throughput():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, world, got, thr in res:
        assert world == 2 and got == 125.0
        assert thr == pytest.approx(2 * 10 / 0.125)


def test_single_rank_needs_no_process_group(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    r = bench.Ranks("gloo")
    assert (r.world, r.rank) == (1, 0)
    r.barrier()
    assert r.max_over_ranks(3.5) == 3.5
    r.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1"])
    a = bench.parse()
    assert bench.run_reference(a) is None
