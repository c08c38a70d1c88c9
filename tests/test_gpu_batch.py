"""Batched solves: several independent instances of different sizes and depths in one tile pool,
solved by one graph launch.  Each instance's result must be bit-identical to the same instance
solved alone (a batch of one) — the reductions are per instance in a fixed order and every other
kernel works tile by tile — and agree with the CPU oracle like a single solve does."""
from __future__ import annotations

import numpy as np
import pytest

from cirrus_b200 import KERNEL_GS_SWEEP, KERNEL_LAPLACIAN, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP, KERNEL_RESIDUAL_RESTRICT, CirrusError, DeviceGrid, GMGSolver, PRECISION_MIXED_FP64, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MIX = ["sphere64_small", "ring64_small", "uniform32_small", "sphere64_neumann_small"]


def rhs_of(b):
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    rhs = g.get_channel(1)
    g.close()
    return rhs


def alone(b, rhs, solver, pure):
    g = DeviceGrid(b.topology)
    g.set_channel(1, rhs)
    it, rel = solver.solve(g, is_pure_neumann=pure)
    x = g.get_channel(0)
    g.close()
    return it, rel, x


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_batch_results_equal_alone(built_cache):
    bs = [built_cache(n) for n in MIX]
    rhs = [rhs_of(b) for b in bs]
    pure = [b.workload.pure_neumann for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    assert g.num_instances == len(bs)
    for i, r in enumerate(rhs):
        g.set_channel_instance(i, 1, r)
    s = GMGSolver()
    # one launch for Dirichlet and pure-Neumann instances together (per-instance flags)
    res = s.solve_batch(g, pure_neumann=pure)
    for i, b in enumerate(bs):
        it, rel = res[i]
        ait, arel, ax = alone(b, rhs[i], GMGSolver(), pure[i])
        x = g.get_channel_instance(i, 0)
        print(f"{MIX[i]}: batch {it} iters {rel:.3e}; alone {ait} iters {arel:.3e}")
        assert (it, rel) == (ait, arel)
        assert np.array_equal(bits(x), bits(ax))
    g.close()


def test_batch_inactive_instance_untouched(built_cache):
    bs = [built_cache(n) for n in ["sphere64_small", "uniform32_small"]]
    g = DeviceGrid([b.topology for b in bs])
    rng = np.random.default_rng(3)
    marker = rng.standard_normal((bs[1].tiles.shape[0], 512)).astype(np.float32)
    g.set_channel_instance(0, 1, rhs_of(bs[0]))
    for ch in (0, 1):
        g.set_channel_instance(1, ch, marker)
    res = GMGSolver().solve_batch(g, active=[True, False])
    assert res[0][1] < 1e-6 and res[0][0] > 0
    assert res[1] == (0, 0.0)
    for ch in (0, 1):
        assert np.array_equal(bits(g.get_channel_instance(1, ch)), bits(marker))
    g.close()


def test_batch_of_same_shape_different_rhs(built_cache):
    b = built_cache("ring64_small")
    rng = np.random.default_rng(11)
    base = rhs_of(b)
    rhs = [base, base * np.float32(0.5), (base + rng.standard_normal(base.shape).astype(np.float32) * np.float32(1e-3) *
                                          (base != 0)).astype(np.float32)]
    g = DeviceGrid([b.topology] * len(rhs))
    for i, r in enumerate(rhs):
        g.set_channel_instance(i, 1, r)
    res = GMGSolver().solve_batch(g)
    for i, r in enumerate(rhs):
        ait, arel, ax = alone(b, r, GMGSolver(), False)
        assert res[i] == (ait, arel)
        assert np.array_equal(bits(g.get_channel_instance(i, 0)), bits(ax))
    g.close()


def test_batch_against_oracle(built_cache):
    """The batched solve agrees with the CPU oracle as a single solve does (iterations within one,
    pressure within 1e-5 relative L2 of the FP32 mirror)."""
    names = ["sphere64_small", "ring64_small"]
    bs = [built_cache(n) for n in names]
    rhs = [rhs_of(b) for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    for i, r in enumerate(rhs):
        g.set_channel_instance(i, 1, r)
    res = GMGSolver().solve_batch(g)
    for i, b in enumerate(bs):
        f = O.CpuOracle(b.tiles)
        f.set_ctypes(b.ctypes)
        f.set_channel_f32(1, rhs[i])
        oit, orel, _ = f.solve(O.CpuOracle.FP32, 1000, 1e-6)
        ox = f.get_channel_f32(0)
        x = g.get_channel_instance(i, 0)
        leaf = (b.tiles[:, 4] & 1).astype(bool)
        err = np.linalg.norm((x[leaf] - ox[leaf]).astype(np.float64)) / np.linalg.norm(ox[leaf].astype(np.float64))
        assert abs(res[i][0] - oit) <= 1
        assert err <= 1e-5
    g.close()


def test_batch_mixed_precision_reaches_1e8(built_cache):
    bs = [built_cache(n) for n in ["sphere64_small", "ring64_small", "uniform32_small"]]
    rhs = [rhs_of(b) for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    for i, r in enumerate(rhs):
        g.set_channel_instance(i, 1, r)
    s = GMGSolver(precision=PRECISION_MIXED_FP64)
    s.solve_batch(g, relative_tolerance=1e-8)
    for i in range(len(bs)):
        assert s.last_results[i].status == 0
        assert s.last_results[i].true_rel_residual < 1e-8
    g.close()


def test_autotune_changes_timing_not_results(built_cache):
    """The launch shapes the autotuner picks compute every tile with the same operations: solves
    before and after tuning are bit-identical (batch and single grids)."""
    bs = [built_cache(n) for n in ["ring64_small", "sphere64_small"]]
    rhs = [rhs_of(b) for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    s = GMGSolver()
    out = []
    for tune in (False, True):
        if tune:
            g.autotune(reps=3)
        for i, r in enumerate(rhs):
            g.set_channel_instance(i, 1, r)
        res = s.solve_batch(g)
        out.append((res, [g.get_channel_instance(i, 0) for i in range(len(bs))]))
    assert out[0][0] == out[1][0]
    for a, b in zip(out[0][1], out[1][1]):
        assert np.array_equal(bits(a), bits(b))
    g.close()


def test_autotune_whole_solve_refinement_restores_b_and_x(built_cache):
    """On a small grid the autotuner also times whole solves of the grid's own right-hand sides;
    it leaves channel 1 (b) and channel 0 (x) as it found them, picks only valid shapes, and the
    solve after tuning gives the untuned solve's bits."""
    b = built_cache("ring512")
    rhs = rhs_of(b)
    g = DeviceGrid(b.topology)
    assert g.get_launch_shape(KERNEL_GS_SWEEP, 6) == 4  # the untuned shape
    s = GMGSolver()
    g.set_channel(1, rhs)
    it0, rel0 = s.solve(g)
    x0 = g.get_channel(0)
    g.set_channel(1, rhs)
    x_marker = np.arange(x0.size, dtype=np.float32).reshape(x0.shape)
    g.set_channel(0, x_marker)
    g.autotune(reps=3)
    assert np.array_equal(bits(g.get_channel(1)), bits(rhs))
    assert np.array_equal(bits(g.get_channel(0)), bits(x_marker))
    for k in (KERNEL_GS_SWEEP, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP, KERNEL_RESIDUAL_RESTRICT):
        for lv in range(2, 7):
            assert 0 <= g.get_launch_shape(k, lv) < 12
    assert 0 <= g.get_launch_shape(KERNEL_LAPLACIAN, 0) < 20
    g.set_channel(0, np.zeros_like(x0))  # the solve writes x on LEAF tiles only; start as the first did
    it1, rel1 = s.solve(g)
    assert (it1, rel1) == (it0, rel0)
    assert np.array_equal(bits(g.get_channel(0)), bits(x0))
    g.close()


@pytest.mark.parametrize("groups", [[["sphere64_small", "ring64_small"], ["ring512"]], [["ring512"], ["ring512", "ring64_small"], ["sphere64_small"]]])
def test_grids_solved_at_once_give_each_grids_bits(built_cache, groups):
    """Several grids solved at once (cirrus_gmg_solve_grids: each grid's graph on its own stream)
    give, grid by grid, the iterations and pressure of that grid's own batched solve bit for bit;
    the same grid twice is refused; mixed precision (one host thread per grid) gives each grid's
    own mixed solve bit for bit."""
    grids, rhs = [], []
    for names in groups:
        bs = [built_cache(n) for n in names]
        rhs.append([rhs_of(b) for b in bs])
        grids.append(DeviceGrid([b.topology for b in bs]))

    def load():
        for g, rs in zip(grids, rhs):
            for i, r in enumerate(rs):
                g.set_channel_instance(i, 1, r)
                g.set_channel_instance(i, 0, np.zeros_like(r))

    s = GMGSolver()
    load()
    alone = []
    for g in grids:
        res = s.solve_batch(g)
        alone.append((res, [g.get_channel_instance(i, 0) for i in range(g.num_instances)]))
    load()
    together = s.solve_grids(grids)
    assert all(r.status == 0 for r in s.last_results)
    for g, (res, xs), res2 in zip(grids, alone, together):
        assert res2 == res
        for i, x in enumerate(xs):
            assert np.array_equal(bits(g.get_channel_instance(i, 0)), bits(x)), i
    with pytest.raises(CirrusError):
        s.solve_grids([grids[0], grids[0]])
    # kernels launched one by one from the host (each grid's loop checked on the host in turn)
    for g in grids:
        g.set_launch_mode(True)
    load()
    direct = s.solve_grids(grids)
    for g, (res, xs), res2 in zip(grids, alone, direct):
        assert res2 == res
        for i, x in enumerate(xs):
            assert np.array_equal(bits(g.get_channel_instance(i, 0)), bits(x)), i
        g.set_launch_mode(False)
    sm = GMGSolver(precision=PRECISION_MIXED_FP64)
    load()
    malone = []
    for g in grids:
        res = sm.solve_batch(g)
        malone.append((res, [g.get_channel_instance(i, 0) for i in range(g.num_instances)]))
    load()
    mtogether = sm.solve_grids(grids)  # one host thread per grid
    assert all(r.status == 0 and r.true_rel_residual < 1e-6 for r in sm.last_results)
    for g, (res, xs), res2 in zip(grids, malone, mtogether):
        assert res2 == res
        for i, x in enumerate(xs):
            assert np.array_equal(bits(g.get_channel_instance(i, 0)), bits(x)), i
    for g in grids:
        g.close()


def test_every_launch_shape_gives_the_same_bits(built_cache):
    """Each of the eight plain launch shapes of the staged kernels (tiles per CTA x tiles in flight),
    pinned for every kernel and level, gives the solve of the default shapes bit for bit."""
    bs = [built_cache(n) for n in ["sphere64_small", "ring64_small"]]
    rhs = [rhs_of(b) for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    s = GMGSolver()
    out = []
    for shape in (None, 0, 1, 2, 3, 4, 5, 6, 7):
        if shape is not None:
            g.set_launch_shape(shape)
            assert g.get_launch_shape(KERNEL_PROLONG_SWEEP, 1) == shape
        for i, r in enumerate(rhs):
            g.set_channel_instance(i, 1, r)
            g.set_channel_instance(i, 0, np.zeros_like(r))
        res = s.solve_batch(g)
        out.append((res, [g.get_channel_instance(i, 0) for i in range(len(bs))]))
    for res, xs in out[1:]:
        assert res == out[0][0]
        for a, b in zip(out[0][1], xs):
            assert np.array_equal(bits(a), bits(b))
    g.close()


@pytest.mark.parametrize("names", [["sphere64_small", "ring64_small"], ["ring512"], ["ring512"] * 4])
def test_tma_and_column_laplacian_shapes_give_the_same_bits(built_cache, names):
    """The Laplacian's TMA-staged pipeline (shapes 8-11: one producer warp issuing bulk tensor
    copies of each tile, its halos and masks into a ring of shared-memory stages, 1-4 consumer
    groups), its eight-cells-per-thread layout (shapes 12-15: 64 threads per tile) and the
    4-cell shapes that prefetch later CTAs' tiles into L2 (shapes 16-19) inside the
    solve -- A p of every LEAF tile, the GHOST rows, the p.Ap tile parts -- give the iterations and
    pressure of the cp.async-staged 4-cell shape bit for bit."""
    bs = [built_cache(n) for n in names]
    rhs = [rhs_of(b) for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    s = GMGSolver()
    out = []
    shapes = (1, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19)
    for shape in shapes:
        g.set_launch_shape(shape, KERNEL_LAPLACIAN)
        assert g.get_launch_shape(KERNEL_LAPLACIAN, 0) == shape
        for i, r in enumerate(rhs):
            g.set_channel_instance(i, 1, r)
            g.set_channel_instance(i, 0, np.zeros_like(r))
        res = s.solve_batch(g)
        assert all(r.status == 0 for r in s.last_results), shape
        out.append((res, [g.get_channel_instance(i, 0) for i in range(len(bs))]))
    for shape, (res, xs) in zip(shapes[1:], out[1:]):
        assert res == out[0][0], shape
        for a, b in zip(out[0][1], xs):
            assert np.array_equal(bits(a), bits(b)), shape
    g.close()


@pytest.mark.parametrize("kernel", [KERNEL_GS_SWEEP, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP, KERNEL_RESIDUAL_RESTRICT])
@pytest.mark.parametrize("names", [["sphere64_small", "ring64_small"], ["ring512"] * 2])
def test_prefetching_stencil_shapes_give_the_same_bits(built_cache, names, kernel):
    """The V-cycle's staged kernels in the shapes that prefetch later CTAs' tiles into L2 (8-11),
    pinned at every level, give the iterations and pressure of shape 1 bit for bit."""
    bs = [built_cache(n) for n in names]
    rhs = [rhs_of(b) for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    s = GMGSolver()
    out = []
    shapes = (1, 8, 9, 10, 11)
    for shape in shapes:
        for lvl in range(int(max(int(b.tiles[:, 0].max()) for b in bs)) + 1):
            g.set_launch_shape(shape, kernel, lvl)
        assert g.get_launch_shape(kernel, 1) == shape
        for i, r in enumerate(rhs):
            g.set_channel_instance(i, 1, r)
            g.set_channel_instance(i, 0, np.zeros_like(r))
        res = s.solve_batch(g)
        assert all(r.status == 0 for r in s.last_results), shape
        out.append((res, [g.get_channel_instance(i, 0) for i in range(len(bs))]))
    for shape, (res, xs) in zip(shapes[1:], out[1:]):
        assert res == out[0][0], shape
        for a, b in zip(out[0][1], xs):
            assert np.array_equal(bits(a), bits(b)), shape
    g.close()


def test_sweep_tuner_picks_a_converging_pair_and_keeps_b(built_cache):
    """The sweep-count tuner returns one of its candidate (level_iters, coarsest_iters) pairs,
    leaves the right-hand sides bit-identical, and the mixed-precision batched solve with that
    pair reaches the FP64 tolerance on every instance."""
    bs = [built_cache(n) for n in ["sphere64_small", "ring64_small"]]
    rhs = [rhs_of(b) for b in bs]
    g = DeviceGrid([b.topology for b in bs])
    for i, r in enumerate(rhs):
        g.set_channel_instance(i, 1, r)
    s = GMGSolver(precision=PRECISION_MIXED_FP64)
    li, ci = s.autotune_sweeps(g)
    assert (li, ci) in {(1, 2), (1, 4), (1, 6), (1, 10), (1, 16), (1, 24), (2, 10)}
    for i, r in enumerate(rhs):
        assert np.array_equal(bits(g.get_channel_instance(i, 1)), bits(r))
    s.solve_batch(g, level_iters=li, coarsest_iters=ci)
    for r in s.last_results:
        assert r.status == 0 and r.true_rel_residual < 1e-6
    g.close()


def test_batch_of_64_random_spheres():
    """The batched configuration: 64 independent instances (64^3-256^3 effective, 1-4 levels,
    1-5 random spheres each) in one mixed-precision batched launch; every instance reaches a 1e-6
    FP64 true relative residual, and sampled instances are bit-identical to their solves alone."""
    bs = [W.build(w) for w in W.batch_of_spheres(64)]
    g = DeviceGrid([b.topology for b in bs])
    for i, b in enumerate(bs):
        for a in range(3):
            g.set_channel_instance(i, 6 + a, b.velocity[a])
    g.projection_rhs()
    rhs = [g.get_channel_instance(i, 1) for i in range(len(bs))]
    s = GMGSolver(precision=PRECISION_MIXED_FP64)
    s.solve_batch(g, relative_tolerance=1e-6)
    res = list(s.last_results)
    assert all(r.status == 0 and r.true_rel_residual < 1e-6 for r in res)
    for i in (0, 17, 63):
        ga = DeviceGrid(bs[i].topology)
        ga.set_channel(1, rhs[i])
        sa = GMGSolver(precision=PRECISION_MIXED_FP64)
        sa.solve(ga, relative_tolerance=1e-6)
        ra = sa.last_result
        assert (ra.iters, ra.outer_iters, ra.true_rel_residual) == (res[i].iters, res[i].outer_iters, res[i].true_rel_residual)
        assert np.array_equal(bits(ga.get_channel(0)), bits(g.get_channel_instance(i, 0)))
        ga.close()
    g.close()
