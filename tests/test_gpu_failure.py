"""Failure detection with host-injected faults: a NaN planted in one instance's right-hand side
(on the host, before upload).  The solver must stop that instance with CIRRUS_ERR_NONFINITE after
its first residual check -- no hang, no endless loop -- and leave every other instance of the
batch bit-identical to the same batch without the fault.  Covers the plain solve, a 4-instance
batch and the mixed-precision (FP64 defect-correction) solve."""
from __future__ import annotations

import numpy as np
import pytest

from cirrus_b200 import DeviceGrid, GMGSolver, PRECISION_MIXED_FP64, workloads as W

pytestmark = pytest.mark.gpu

NONFINITE = 6
MIX = ["sphere64_small", "ring64_small", "uniform32_small", "sphere64_neumann_small"]


def rhs_of(b):
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    rhs = g.get_channel(1)
    g.close()
    return rhs


def poisoned(b, rhs):
    """A copy of rhs with one INTERIOR cell of a LEAF tile set to NaN."""
    out = rhs.copy()
    leaf = np.flatnonzero((b.tiles[:, 4] & W.LEAF) != 0)
    t = int(leaf[len(leaf) // 2])
    c = int(np.flatnonzero(b.ctypes[t] & W.INTERIOR)[0])
    out[t, c] = np.nan
    return out


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_nan_plain_solve_stops_and_grid_stays_usable(built_cache):
    b = built_cache("sphere64_small")
    rhs = rhs_of(b)
    g = DeviceGrid(b.topology)
    s = GMGSolver()
    g.set_channel(1, poisoned(b, rhs))
    it, rel = s.solve(g)
    assert s.last_result.status == NONFINITE
    assert it <= 1 and not np.isfinite(rel)
    # the same grid afterwards: a clean solve converges with the bits of a fresh grid
    g.set_channel(1, rhs)
    it2, rel2 = s.solve(g)
    assert s.last_result.status == 0 and rel2 < 1e-6
    x2 = g.get_channel(0)
    g.close()
    g3 = DeviceGrid(b.topology)
    g3.set_channel(1, rhs)
    it3, rel3 = GMGSolver().solve(g3)
    assert (it2, rel2) == (it3, rel3)
    assert np.array_equal(bits(x2), bits(g3.get_channel(0)))
    g3.close()


@pytest.mark.parametrize("precision", [0, PRECISION_MIXED_FP64])
def test_nan_in_one_batch_instance(built_cache, precision):
    bs = [built_cache(n) for n in MIX]
    rhs = [rhs_of(b) for b in bs]
    pure = [b.workload.pure_neumann for b in bs]
    bad = 1

    def run(rs):
        g = DeviceGrid([b.topology for b in bs])
        for i, r in enumerate(rs):
            g.set_channel_instance(i, 1, r)
        s = GMGSolver(precision=precision)
        s.solve_batch(g, pure_neumann=pure)
        res = [(r.iters, r.rel_residual, r.status) for r in s.last_results]
        xs = [g.get_channel_instance(i, 0) for i in range(len(bs))]
        g.close()
        return res, xs

    clean, xc = run(rhs)
    faulty, xf = run([poisoned(bs[i], r) if i == bad else r for i, r in enumerate(rhs)])
    print("clean", clean)
    print("faulty", faulty)
    assert faulty[bad][2] == NONFINITE
    for i in range(len(bs)):
        if i == bad:
            continue
        assert clean[i][2] == 0 and faulty[i] == clean[i], MIX[i]
        assert np.array_equal(bits(xf[i]), bits(xc[i])), MIX[i]
