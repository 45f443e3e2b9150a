"""The multi-rank (replicas only) path of bench.py on CPU: two gloo ranks.
Each rank builds its own seeded system, the step timings are reduced to
their maximum over the ranks, and the reference arm runs on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws)
    try:
        ws_, rk, lr = bench.dist_env()
        assert (ws_, rk, lr) == (ws, rank, rank)
        times = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * rank], ws, device="cpu")
        sysm = bench.make_sys("w2", bench.replica_seed(2024, rank))
        out[rank] = (times, sysm.pos.copy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replicas_and_max_timing():
    ws = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(ws, _free_port(), out), nprocs=ws, join=True)
    t0, p0 = out[0]
    t1, p1 = out[1]
    assert t0 == t1 == [2.0, 10.0, 0.5]
    # replicas: each rank has its own seeded system
    assert p0.shape == p1.shape and (p0 != p1).any()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(bench.parse()) == 0
