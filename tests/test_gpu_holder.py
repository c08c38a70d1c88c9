"""Tile-holder files between the product and the reference build, on the GPU: a holder the
reference writes from its own grid (getHostTileHolder + its file layout) is read by the product
with the reference's tiles, channels and cell types bit for bit; a holder the product writes from
its device grid is read back by the reference (setTilesFromHolder + compressHost) into the same
tiles, hash order, cell types and channels; and a holder is a warm start for the next solve."""
from __future__ import annotations

import numpy as np
import pytest

from cirrus_b200 import DeviceGrid, GMGSolver, Holder, PRECISION_MIXED_FP64, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ALL = W.LEAF | W.NONLEAF | W.GHOST


@pytest.fixture(scope="module")
def ref_ok():
    if not O.ref_available():
        pytest.skip("reference build oracle/_ref/libcirrus_ref.so not present")
    return True


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def ref_grid(b):
    w = b.workload
    ref = O.RefHarness(w)
    ref.calc_neighbors()
    ref.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    return ref


@pytest.mark.parametrize("name", ["sphere64_small", "ring64_small", "ring512"])
@pytest.mark.parametrize("types", [ALL, W.LEAF])
def test_reference_holder_read_by_product(tmp_path, built_cache, ref_ok, name, types):
    b = built_cache(name)
    ref = ref_grid(b)
    ref.rhs(b.velocity)
    ref.solve(1000, 1e-6, 1, 10, 1, b.workload.pure_neumann)
    p = tmp_path / "ref.bin"
    ref.write_holder(p, types)
    h = Holder.read(p)
    sel = (b.tiles[:, 4] & types) != 0
    assert np.array_equal(h.tiles(), b.tiles[sel])
    assert np.array_equal(h.cell_types(), ref.ctypes()[sel])
    for c in (0, 1, 6, 7, 8):
        assert np.array_equal(bits(h.channel(c)), bits(ref.get_channel(c)[sel])), c
    if types == ALL:
        topo, order = h.to_topology(b.workload.log2_hash)
        assert np.array_equal(topo.tiles(), b.tiles)
        assert np.array_equal(topo.hash_slots(), b.topology.hash_slots())


@pytest.mark.parametrize("name", ["sphere64_small", "ring64_small", "ring512"])
def test_product_holder_read_by_reference(tmp_path, built_cache, ref_ok, name):
    b = built_cache(name)
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    GMGSolver().solve(g, is_pure_neumann=b.workload.pure_neumann)
    p = tmp_path / "ours.bin"
    Holder.from_grid(b.topology, g, ALL).write(p)
    ref = O.RefHarness.from_holder(p, b.workload.log2_hash)
    assert np.array_equal(ref.tiles(), b.tiles)
    assert np.array_equal(ref.slots(), b.topology.hash_slots())
    assert np.array_equal(ref.ctypes(), b.ctypes)
    for c in (0, 1, 6):
        assert np.array_equal(bits(ref.get_channel(c)), bits(g.get_channel(c))), c
    g.close()


def test_holder_as_warm_start(tmp_path, built_cache):
    """Checkpoint the pressure of a solve to a holder, restart from the file into a new grid and
    solve the next (slightly changed) right-hand side from it: fewer iterations than from zero,
    the same FP64 tolerance reached."""
    b = built_cache("ring64_small")
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    rhs = g.get_channel(1)
    s = GMGSolver(precision=PRECISION_MIXED_FP64)
    s.solve(g, relative_tolerance=1e-8)
    assert s.last_result.status == 0
    p = tmp_path / "ckpt.bin"
    Holder.from_grid(b.topology, g, ALL).write(p)
    g.close()

    h = Holder.read(p)
    topo, order = h.to_topology(b.workload.log2_hash)
    rng = np.random.default_rng(1)
    nxt = (rhs * (1 + np.float32(1e-4) * rng.standard_normal(rhs.shape).astype(np.float32))).astype(np.float32)
    runs = {}
    for warm in (False, True):
        g2 = DeviceGrid(topo)
        if warm:
            h.load_into(g2, order, channels=(0,))
        g2.set_channel(1, nxt)
        s2 = GMGSolver(precision=PRECISION_MIXED_FP64, warm_start=warm)
        s2.solve(g2, relative_tolerance=1e-8)
        r = s2.last_result
        runs[warm] = (r.iters, r.status, r.true_rel_residual)
        g2.close()
    print(runs)
    assert runs[True][1] == 0 and runs[False][1] == 0
    assert runs[True][2] < 1e-8 and runs[False][2] < 1e-8
    assert runs[True][0] < runs[False][0]
