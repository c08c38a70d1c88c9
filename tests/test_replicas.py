"""The multi-GPU path is replicas only: every rank solves its own instances (disjoint seeds) with
no collective on the data path; the only collectives are the barrier and the max of the ranks'
times that bench.py reports.  Exercised here with two gloo ranks on the CPU, each solving its
instance with the CPU oracle."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    sys.path.insert(0, str(ROOT))
    import datetime
    import time

    import numpy as np
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                            timeout=datetime.timedelta(seconds=60))
    import bench
    from cirrus_b200 import workloads as W
    from oracle import oracle as O

    seeds = bench.batch_seeds(rank, 3)
    w = W.make("uniform32_small", seeds[0])
    b = W.build(w)
    # the rank's own seeded right-hand side on its INTERIOR leaf cells
    f = O.CpuOracle(b.tiles)
    f.set_ctypes(b.ctypes)
    rng = np.random.default_rng(seeds[0])
    leaf = (b.tiles[:, 4] & 1) != 0
    rhs = np.where(leaf[:, None] & ((b.ctypes & 2) != 0), rng.standard_normal(b.ctypes.shape), 0).astype(np.float32)
    t0 = time.perf_counter()
    f.set_channel_f32(1, rhs)
    it, rel, _ = f.solve(O.CpuOracle.FP32, 1000, 1e-6)
    dt = time.perf_counter() - t0 + 0.25 * rank  # ranks finish at different times
    m = bench.barrier_max(dist, dt)
    q.put((rank, seeds, dt, m, it, rel))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, t0, m0, it0, rel0), (r1, s1, t1, m1, it1, rel1) = out
    assert set(s0).isdisjoint(s1)
    assert m0 == m1 == pytest.approx(max(t0, t1))
    assert rel0 < 1e-6 and rel1 < 1e-6 and it0 > 0 and it1 > 0
