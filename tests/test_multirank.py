"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the job time is
the maximum over ranks, both ranks take the same collective steps, and the
reference arm does its work on rank 0 only. The force path itself runs one
independent replica per GPU (no data-path collective), so these are the only
cross-rank steps."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        dev = torch.device("cpu")
        # the slowest rank sets the job time; every rank learns it
        out[rank] = bench.max_over_ranks(torch, dist, 1.5 + rank, dev)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, None, 3.25, torch.device("cpu")) == 3.25


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"workload": "clustered256", "steps": 1, "warmup": 0})()
    assert bench.run_reference(args) == 0
