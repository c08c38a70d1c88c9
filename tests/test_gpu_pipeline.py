"""The asynchronous end-to-end solve (cirrus_gmg_solve_host_submit / wait): two grids of the same
batch alternating on two streams return the pressures and results of the synchronous call, bit
for bit, and a second submit on a busy grid first completes the one in flight."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from cirrus_b200 import B_CHANNEL, DeviceGrid, GMGSolver, workloads as W

pytestmark = pytest.mark.gpu


def batch(b, seeds):
    g = DeviceGrid([b.topology] * len(seeds))
    for i, sd in enumerate(seeds):
        vel = W.face_velocity(b.tiles, sd)
        for a in range(3):
            g.set_channel_instance(i, 6 + a, vel[a])
    g.projection_rhs()
    return g


@pytest.mark.parametrize("name", ["sphere64_small", "ring64_small"])
def test_pipelined_host_solves_match_synchronous(name, built_cache):
    b = built_cache(name)
    seeds = [3, 4, 5]
    ga, gb = batch(b, seeds), batch(b, seeds)
    rhs = ga.get_channel(B_CHANNEL)
    solver = GMGSolver()
    sync_res = solver.solve_batch(ga)  # per-instance results of the synchronous solve
    ga.set_channel(B_CHANNEL, rhs)
    rhs = rhs.reshape(-1)
    x_ref = np.empty_like(rhs)
    it0, rel0 = solver.solve_host(ga, rhs, x_ref)
    assert (it0, rel0) == sync_res[0]
    b_pin = [torch.from_numpy(rhs.copy()).pin_memory() for _ in range(2)]
    x_pin = [torch.empty_like(b_pin[0]).pin_memory() for _ in range(2)]
    s2 = torch.cuda.Stream()
    grids, streams = [ga, gb], [torch.cuda.current_stream().cuda_stream, s2.cuda_stream]
    for step in range(5):
        j = step % 2
        if step >= 2:
            res = solver.solve_host_wait(grids[j])
            assert res == sync_res
            assert np.array_equal(x_pin[j].numpy().view(np.uint32), x_ref.view(np.uint32))
            x_pin[j].fill_(float("nan"))
        solver.solve_host_submit(grids[j], b_pin[j].numpy(), x_pin[j].numpy(), stream=streams[j])
    # a second submit on a grid with a solve in flight completes the first one
    solver.solve_host_submit(grids[0], b_pin[0].numpy(), x_pin[0].numpy(), stream=streams[0])
    for j in (0, 1):
        res = solver.solve_host_wait(grids[j])
        assert res == sync_res
        assert np.array_equal(x_pin[j].numpy().view(np.uint32), x_ref.view(np.uint32))
