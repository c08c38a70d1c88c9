"""The device-resident topology (RefineLeafsOneStep, CoarsenStep, SpawnGhostTiles,
compressHost/syncHostAndDevice, CalcCellTypesFromLeafs on the GPU) against the host topology
(itself pinned to the reference's golden digests) and against the reference build step by step:
the same tiles in the same hash-slot order, the same hash slots, the same tile status words and
cell types, also through coarsening (removeTileHost's backward-shift deletion) and refinement
after it."""
from __future__ import annotations

import numpy as np
import pytest

from cirrus_b200 import DeviceGrid, DeviceTopology, GMGSolver, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def dev_build(w):
    d = DeviceTopology(w.h0, w.log2_hash)
    d.set_tiles(0, np.array(w.roots, dtype=np.int32), W.LEAF)
    d.compress()
    d.spawn_ghost_tiles()
    d.iterative_refine(w.masks)
    return d


@pytest.mark.parametrize("name", ["uniform32_small", "sphere64_small", "ring64_small", "uniform128", "sphere256", "ring512"])
def test_device_topology_equals_host(name, built_cache):
    b = built_cache(name)
    d = dev_build(b.workload)
    assert np.array_equal(d.tiles(), b.tiles)
    assert np.array_equal(d.hash_slots(), b.topology.hash_slots())
    assert d.max_level == b.topology.max_level
    d.set_cell_types(W.leaf_cell_types(b.workload, b.tiles, b.nbr6))
    d.calc_cell_types_from_leafs()
    assert np.array_equal(d.cell_types(), b.ctypes)


def _ref_ok():
    if not O.ref_available():
        pytest.skip("reference build oracle/_ref/libcirrus_ref.so not present")


def _coarsen_masks(w, tiles, frac):
    """Per level: LEAF tiles of the finest level in the lower `frac` of x get target level - 1."""
    masks = [None] * w.num_layers
    lmax = int(tiles[:, 0].max())
    ext = [e << lmax for e in w.root_extent]
    m = np.zeros(ext, dtype=np.uint8)
    m[: max(1, int(ext[0] * frac))] = 1
    masks[lmax] = m
    return masks


@pytest.mark.parametrize("name", ["sphere64_small", "ring64_small", "ring512"])
def test_device_topology_steps_against_reference(name, built_cache):
    """Every step of the construction compared with the reference's: after each RefineLeafsOneStep
    and each SpawnGhostTiles the tiles, hash slots and status words; then two CoarsenSteps and a
    refinement back, with the deleted-tile counts."""
    _ref_ok()
    b = built_cache(name)
    w = b.workload
    ref = O.RefHarness.roots(w)
    d = DeviceTopology(w.h0, w.log2_hash)
    d.set_tiles(0, np.array(w.roots, dtype=np.int32), W.LEAF)
    d.compress()
    d.spawn_ghost_tiles()

    def same(tag):
        assert np.array_equal(d.tiles(), ref.tiles()), tag
        assert np.array_equal(d.hash_slots(), ref.slots()), tag
        assert np.array_equal(d.statuses(), ref.statuses()), tag

    same("roots")
    for step in range(16):
        rc = d.refine_leafs_one_step(w.masks)
        rr = ref.refine_one_step(w.masks)
        assert rc == rr, step
        same(f"refine {step}")
        d.spawn_ghost_tiles()
        ref.spawn_ghosts()
        same(f"spawn {step}")
        if sum(rc) == 0:
            break
    assert np.array_equal(d.tiles(), b.tiles)
    for k, frac in enumerate((0.5, 0.75)):
        cm = _coarsen_masks(w, d.tiles(), frac)
        dc = d.coarsen_step(cm)
        rc = ref.coarsen_step(cm)
        print(f"{name} coarsen {k}: deleted {dc}")
        assert dc == rc and sum(dc) > 0
        same(f"coarsen {k}")
    # refine back after the deletions (insertion into tables with removed entries)
    for step in range(16):
        rc = d.refine_leafs_one_step(w.masks)
        rr = ref.refine_one_step(w.masks)
        assert rc == rr
        d.spawn_ghost_tiles()
        ref.spawn_ghosts()
        same(f"refine back {step}")
        if sum(rc) == 0:
            break


@pytest.mark.parametrize("name", ["sphere64_small", "ring512"])
def test_grid_from_device_topology_solves_like_host(name, built_cache):
    b = built_cache(name)
    d = dev_build(b.workload)
    d.set_cell_types(W.leaf_cell_types(b.workload, b.tiles, b.nbr6))
    d.calc_cell_types_from_leafs()
    topo = d.to_topology()
    res = []
    for t in (topo, b.topology):
        g = DeviceGrid(t)
        for a in range(3):
            g.set_channel(6 + a, b.velocity[a])
        g.projection_rhs()
        it, rel = GMGSolver().solve(g, is_pure_neumann=b.workload.pure_neumann)
        res.append((it, rel, g.get_channel(0).tobytes()))
        g.close()
    assert res[0] == res[1]
