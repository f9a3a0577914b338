"""The multi-GPU path of the benchmark is replicas only: each rank evaluates
its own theta points and the job's time is the slowest rank's.  Two gloo
ranks on the CPU exercise that logic (rank-distinct points, the max-over-
ranks reduction, the whole-job rate) without a GPU."""
import os
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    sys.path.insert(0, REPO)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        theta = bench.replica_theta([-1.0, 1.0, 0.0, 2.0], rank)
        pts = bench.step_points(theta, 0, 3)
        t_local = 1.0 + rank  # rank 1 is the slow one
        t_max = bench.max_over_ranks(t_local, world)
        out[rank] = (theta.tolist(), [p.tolist() for p in pts], t_max, bench.job_rate(3 * 5, world, t_max))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    th0, pts0, tmax0, rate0 = out[0]
    th1, pts1, tmax1, rate1 = out[1]
    assert not np.allclose(th0, th1)  # independent points per rank
    assert len(pts0) == 3 and not np.allclose(pts0[0], pts0[1])
    assert tmax0 == tmax1 == 2.0  # slowest rank
    assert rate0 == rate1 == 3 * 5 * 2 / 2.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, REPO)
    import types

    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "cpu_sample", lambda *a, **k: called.append(1) or (1.0, ""))
    args = types.SimpleNamespace(warmup=1, steps=1, workload="gst_300x10", cpu_nt=2, gpus=2)
    assert bench.run_reference(args) == 0 and not called
