"""The product against the reference's own CUDA build run on the same GPU, same inputs:
topology bit-exact, right-hand side and Laplacian bit-exact, V-cycle and solve within the
stated tolerances (iterations within one, pressure 1e-5 relative L2)."""
from __future__ import annotations

import numpy as np
import pytest

from cirrus_b200 import DeviceGrid, GMGSolver, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NAMES = ["uniform32_small", "sphere64_small", "sphere64_neumann_small", "ring64_small", "uniform128", "sphere256", "ring512"]


@pytest.fixture(scope="module")
def ref_ok():
    if not O.ref_available():
        pytest.skip("reference build oracle/_ref/libcirrus_ref.so not present")
    return True


def rel_l2(a, ref, mask):
    a = a[mask].astype(np.float64)
    r = ref[mask].astype(np.float64)
    return float(np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-300))


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", NAMES)
def test_against_reference(name, built_cache, ref_ok):
    b = built_cache(name)
    w = b.workload
    ref = O.RefHarness(w)
    # topology, hash layout, neighbours, cell types
    assert np.array_equal(ref.tiles(), b.tiles)
    assert np.array_equal(ref.slots(), b.topology.hash_slots())
    ref.calc_neighbors()
    assert np.array_equal(ref.neighbors(), b.nbr6)
    ref.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    assert np.array_equal(ref.ctypes(), b.ctypes)
    # right-hand side
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    rhs = g.get_channel(1)
    rrhs = ref.rhs(b.velocity)
    # the divergence writes LEAF and GHOST tiles; NONLEAF tiles keep whatever the channel held
    lg = (b.tiles[:, 4] & (W.LEAF | W.GHOST)) != 0
    assert np.array_equal(bits(rhs)[lg], bits(rrhs)[lg])
    # FullNegativeLaplacian
    g.set_channel(2, rhs)
    g.full_negative_laplacian(2, 3)
    ref.set_channel(2, rhs)
    ref.full_lap(2, 3)
    ap, rap = g.get_channel(3), ref.get_channel(3)
    assert np.array_equal(bits(ap)[lg], bits(rap)[lg])
    # V-cycle
    g.set_channel(1, rhs)
    g.vcycle(4, 1, 3, 1, 10)
    ref.set_channel(1, rhs)
    ref.vcycle(4, 1, 3, 1, 10)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    z, rz = g.get_channel(4), ref.get_channel(4)
    vc_bitwise = float((bits(z)[leaf] == bits(rz)[leaf]).mean())
    assert rel_l2(z, rz, leaf) <= 1e-6
    # solve as FluidEuler::project calls it
    g.set_channel(1, rhs)
    it, rel = GMGSolver().solve(g, False, 1000, 1e-6, 1, 10, 1, w.pure_neumann)
    ref.set_channel(1, rhs)
    rit, rrel, ms = ref.solve(1000, 1e-6, 1, 10, 1, w.pure_neumann)
    x, rx = g.get_channel(0), ref.get_channel(0)
    err = rel_l2(x, rx, leaf)
    print(f"{name}: iters {it}/{rit} rel {rel:.3e}/{rrel:.3e} x_rel_l2 {err:.2e} vcycle_bitwise {vc_bitwise:.4f} ref_ms {ms:.2f}")
    assert abs(it - rit) <= 1
    assert err <= 1e-5


def _ref_grid(b):
    w = b.workload
    ref = O.RefHarness(w)
    ref.calc_neighbors()
    ref.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    return ref


def _ref_then_dropin(ref, velocity, pure_neumann):
    """The reference's own solve, then the drop-in (fresh solver object, as FluidEuler::project
    constructs one per call) on the same grid and right-hand side: both results."""
    rhs = ref.rhs(velocity)
    it, rel, _ = ref.solve(1000, 1e-6, 1, 10, 1, pure_neumann)
    x_ref, r_ref = ref.get_channel(0), ref.get_channel(1)
    ref.set_channel(1, rhs)
    ref.set_channel(0, np.zeros_like(rhs))
    dit, drel, dms = ref.solve_dropin(1000, 1e-6, 1, 10, 1, pure_neumann)
    return (it, rel, x_ref, r_ref), (dit, drel, ref.get_channel(0), ref.get_channel(1), dms)


@pytest.mark.parametrize("name", ["sphere64_small", "ring64_small", "ring512"])
def test_dropin_in_reference_grid(name, built_cache, ref_ok):
    """include/cirrus_gmg_dropin.hpp on the reference's own HADeviceGrid: what FluidEuler::project
    runs after switching the solver class -- same iterations, same pressure and residual channels,
    with a fresh solver object per call (the bound pool is found in the drop-in's registry)."""
    b = built_cache(name)
    w = b.workload
    ref = _ref_grid(b)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    for call in range(2):
        (it, rel, x_ref, r_ref), (dit, drel, x_d, r_d, dms) = _ref_then_dropin(ref, b.velocity, w.pure_neumann)
        print(f"{name} call {call}: reference {it} iters {rel:.3e}; drop-in {dit} iters {drel:.3e} ({dms:.2f} ms)")
        assert dit == it and abs(drel - rel) <= 1e-12 * rel  # FP64 sums in another order; x and r bitwise below
        assert np.array_equal(bits(x_d)[leaf], bits(x_ref)[leaf])
        assert np.array_equal(bits(r_d)[leaf], bits(r_ref)[leaf])


def test_dropin_autotune_keeps_the_reference_bits(built_cache, ref_ok):
    """cirrus_dropin::autotune tunes the launch shapes of the pool bound to the reference's grid
    (on the grid's right-hand sides in channel 1); the drop-in's solves after it still give the
    reference's iterations and bits."""
    b = built_cache("ring512")
    w = b.workload
    ref = _ref_grid(b)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    ref.set_channel(1, ref.rhs(b.velocity))
    ref.autotune_dropin()
    (it, rel, x_ref, r_ref), (dit, drel, x_d, r_d, dms) = _ref_then_dropin(ref, b.velocity, w.pure_neumann)
    print(f"tuned drop-in: {dit} iters ({dms:.2f} ms), reference {it}")
    assert dit == it and abs(drel - rel) <= 1e-12 * rel
    assert np.array_equal(bits(x_d)[leaf], bits(x_ref)[leaf])
    assert np.array_equal(bits(r_d)[leaf], bits(r_ref)[leaf])


@pytest.mark.parametrize("name", ["sphere64_small", "ring512"])
def test_dropin_follows_cell_type_changes(name, built_cache, ref_ok):
    """CalcCellTypesFromLeafs rewrites the cell types every step (src/FluidEuler.h:934) without
    changing tiles.  Between solves on the same tiles, a block of INTERIOR cells becomes NEUMANN
    (an obstacle appears), then INTERIOR again: each time the drop-in, a fresh solver object per
    call, gives the reference's iterations and bits, so it never solves with stale masks."""
    b = built_cache(name)
    w = b.workload
    ref = _ref_grid(b)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    base = W.leaf_cell_types(w, b.tiles, b.nbr6)
    # a 4x4x4 block of INTERIOR cells in the LEAF tile nearest the middle of the LEAF list
    cand = [t for t in np.flatnonzero(leaf) if (base[t].reshape(8, 8, 8)[2:6, 2:6, 2:6] == W.INTERIOR).all()]
    assert cand
    t = cand[len(cand) // 2]
    moved = base.copy()
    blk = moved[t].reshape(8, 8, 8)
    blk[2:6, 2:6, 2:6] = W.NEUMANN
    iters = []
    for ct in (base, moved, base):
        ref.set_ctypes(ct)
        ref.calc_cell_types()
        (it, rel, x_ref, r_ref), (dit, drel, x_d, r_d, _) = _ref_then_dropin(ref, b.velocity, w.pure_neumann)
        assert dit == it and abs(drel - rel) <= 1e-12 * rel  # FP64 sums in another order; x and r bitwise below
        assert np.array_equal(bits(x_d)[leaf], bits(x_ref)[leaf])
        assert np.array_equal(bits(r_d)[leaf], bits(r_ref)[leaf])
        iters.append(it)
        # the obstacle's cells carry no pressure in the moved case
        assert (x_ref[t].reshape(8, 8, 8)[2:6, 2:6, 2:6] == 0).all() == (ct is moved)
    print(f"{name}: iterations {iters} (tile {t} block NEUMANN in the second solve)")


def test_dropin_registry_rebinds_on_new_tiles(built_cache, ref_ok):
    """Two reference grids solved alternately through fresh drop-in objects: each keeps its own
    pool in the registry and gives the reference's bits; release_all frees both."""
    bs = [built_cache("sphere64_small"), built_cache("ring64_small")]
    refs = [_ref_grid(b) for b in bs]
    O.ref_dropin_lib().refdrop_release_all()
    for _ in range(2):
        for b, ref in zip(bs, refs):
            leaf = (b.tiles[:, 4] & W.LEAF) != 0
            (it, rel, x_ref, _), (dit, drel, x_d, _, _) = _ref_then_dropin(ref, b.velocity, b.workload.pure_neumann)
            assert dit == it and abs(drel - rel) <= 1e-12 * rel  # FP64 sums in another order; x and r bitwise below
            assert np.array_equal(bits(x_d)[leaf], bits(x_ref)[leaf])
    assert O.ref_dropin_lib().refdrop_bound_grids() == 2
    O.ref_dropin_lib().refdrop_release_all()
    assert O.ref_dropin_lib().refdrop_bound_grids() == 0


@pytest.mark.parametrize("name", ["uniform32_small", "sphere64_small", "sphere64_neumann_small", "ring64_small", "ring512"])
def test_gradient_against_reference_and_oracle(name, built_cache, ref_ok):
    """AddGradientToFaceCenters, the step after the solve in FluidEuler::project: the product,
    the reference build and the CPU oracle agree bit for bit on the updated face velocities and
    the pressure propagated to GHOST cells, for a solved pressure and a seeded velocity."""
    b = built_cache(name)
    w = b.workload
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    GMGSolver().solve(g, is_pure_neumann=w.pure_neumann)
    p = g.get_channel(0)
    rng = np.random.default_rng(5)
    u = [rng.standard_normal(p.shape).astype(np.float32) for _ in range(3)]
    for a in range(3):
        g.set_channel(6 + a, u[a])
    g.add_gradient_to_face_centers(0, 6)
    gp, gu = g.get_channel(0), [g.get_channel(6 + a) for a in range(3)]

    ref = O.RefHarness(w)
    ref.calc_neighbors()
    ref.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    rp, ru = ref.add_gradient(p, u)

    f = O.CpuOracle(b.tiles)
    f.set_ctypes(b.ctypes)
    op, ou = f.add_gradient(p, u)

    ghost = (b.tiles[:, 4] & W.GHOST) != 0
    assert np.array_equal(bits(gp)[ghost], bits(rp)[ghost])
    assert np.array_equal(bits(op)[ghost], bits(rp)[ghost])
    for a in range(3):
        assert np.array_equal(bits(gu[a]), bits(ru[a])), f"axis {a}: product vs reference"
        assert np.array_equal(bits(ou[a]), bits(ru[a])), f"axis {a}: oracle vs reference"
    g.close()


@pytest.mark.parametrize("name", ["uniform32_small", "sphere64_small", "ring64_small"])
def test_damped_jacobi_against_reference_and_oracle(name, built_cache, ref_ok):
    """GMGSolver::dampedJacobiSolve, the reference's other public solver: the product, the
    reference build, the drop-in header on the reference grid and the CPU oracle take the same
    number of iterations and leave x, the residual and the diagonal bit-identical on LEAF cells."""
    b = built_cache(name)
    w = b.workload
    ref = _ref_grid(b)
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    rhs = g.get_channel(1)
    o = O.CpuOracle(b.tiles)
    o.set_ctypes(b.ctypes)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    omega = float(np.float32(2.0 / 3.0))
    ref.set_channel(1, rhs)
    _, rel5 = ref.damped_jacobi(5, 1e-9, omega)
    for max_iters, tol in ((20, 1e-9), (100, rel5 * (1 + 1e-9))):
        ref.set_channel(1, rhs)
        rit, rrel = ref.damped_jacobi(max_iters, tol, omega)
        rch = [ref.get_channel(c) for c in (0, 2, 3)]
        g.set_channel(1, rhs)
        it, rel = GMGSolver().damped_jacobi_solve(g, False, max_iters, tol, omega)
        ch = [g.get_channel(c) for c in (0, 2, 3)]
        o.set_channel_f32(1, rhs)
        oit, orel = o.damped_jacobi(O.CpuOracle.FP32, max_iters, tol, omega)
        och = [o.get_channel_f32(c) for c in (0, 2, 3)]
        dit, drel = ref.damped_jacobi_dropin(max_iters, tol, omega)
        dch = [ref.get_channel(c) for c in (0, 2, 3)]
        print(f"{name} max_iters {max_iters}: iters {it}/{rit}/{oit}/{dit} rel {rel:.6e}/{rrel:.6e}/{orel:.6e}/{drel:.6e}")
        assert it == rit == oit == dit
        assert rit <= (4 if max_iters == 100 else 20)
        for r in (rel, orel, drel):
            assert abs(r - rrel) <= 1e-12 * rrel
        for c, a, rr, ro, d in zip((0, 2, 3), ch, rch, och, dch):
            assert np.array_equal(bits(a)[leaf], bits(rr)[leaf]), f"channel {c} vs reference"
            assert np.array_equal(bits(ro)[leaf], bits(a)[leaf]), f"channel {c} vs oracle"
            assert np.array_equal(bits(d)[leaf], bits(a)[leaf]), f"channel {c} drop-in"


@pytest.mark.parametrize("name", ["uniform32_small", "sphere64_small", "ring64_small", "sphere256"])
def test_laplacian_variants_against_reference(name, built_cache, ref_ok):
    """FullNegativeLaplacian(calc_diag = true) and NegativeLaplacianSameLevel128 against the
    reference's own kernels on its grid: same bits on every tile, computed or untouched."""
    from test_gpu_kernels import same_level_cases

    b = built_cache(name)
    w = b.workload
    ref = O.RefHarness(w)
    ref.calc_neighbors()
    ref.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    g = DeviceGrid(b.topology)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((b.n, 512)).astype(np.float32)
    y0 = rng.standard_normal((b.n, 512)).astype(np.float32)
    lg = (b.tiles[:, 4] & (W.LEAF | W.GHOST)) != 0
    for diag in (False, True):
        g.set_channel(2, x)
        g.full_negative_laplacian(2, 3, calc_diag=diag)
        ref.set_channel(2, x)
        ref.full_lap_ex(2, 3, diag)
        assert np.array_equal(bits(g.get_channel(3))[lg], bits(ref.get_channel(3))[lg]), diag
    for case in same_level_cases(int(b.tiles[:, 0].max())):
        g.set_channel(2, x)
        g.set_channel(3, y0)
        g.negative_laplacian_same_level(*case[:3], 2, 3, bool(case[3]))
        ref.set_channel(2, x)
        ref.set_channel(3, y0)
        ref.lap_same_level(*case[:3], 2, 3, bool(case[3]))
        assert np.array_equal(bits(g.get_channel(3)), bits(ref.get_channel(3))), case


@pytest.mark.parametrize("name", ["sphere64_small", "sphere64_neumann_small"])
def test_stopping_rules_against_reference(name, built_cache, ref_ok):
    """GMGSolver::solve's stopping rules (src/GMGSolver.cu:546-551, 612-628, 660-665): an iteration
    cap reached before convergence, no convergence checks at all (sync_stride 0: max_iters
    iterations, relative residual -1), and checks every third iteration -- same iteration count,
    same returned residual, and the pressure of the reference build."""
    b = built_cache(name)
    w = b.workload
    ref = O.RefHarness(w)
    ref.calc_neighbors()
    ref.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    ref.calc_cell_types()
    ref.calc_neighbors()
    rhs = ref.rhs(b.velocity)
    g = DeviceGrid(b.topology)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    for max_iters, sync_stride in ((3, 1), (5, 0), (1000, 3)):
        ref.set_channel(1, rhs)
        rit, rrel, _ = ref.solve(max_iters, 1e-6, 1, 10, sync_stride, w.pure_neumann)
        g.set_channel(1, rhs)
        it, rel = GMGSolver().solve(g, False, max_iters, 1e-6, 1, 10, sync_stride, w.pure_neumann)
        x, rx = g.get_channel(0), ref.get_channel(0)
        same = float((bits(x)[leaf] == bits(rx)[leaf]).mean())
        print(f"{name} max_iters {max_iters} sync_stride {sync_stride}: iters {it}/{rit} rel {rel:.6e}/{rrel:.6e} "
              f"x bitwise {same:.4f}")
        assert it == rit
        assert rel == rrel if sync_stride <= 0 else abs(rel - rrel) <= 1e-9 * abs(rrel)
        assert rel_l2(x, rx, leaf) <= 1e-6


def test_dropin_time_at_call_site(built_cache, ref_ok):
    """The drop-in's cost where FluidEuler::project pays it: ring512, one solve per call, a fresh
    solver object per call (src/FluidEuler.h:591), host clock around the call as the reference
    times it (src/FluidEuler.h:595-601).  The first call binds the grid (reads the cell types,
    builds the pool and the graph); later calls find the pool in the registry and only check the
    cell types on the device.  Prints the reference's time beside it."""
    b = built_cache("ring512")
    w = b.workload
    ref = _ref_grid(b)
    rhs = ref.rhs(b.velocity)
    O.ref_dropin_lib().refdrop_release_all()
    ref_ms, drop_ms = [], []
    for i in range(6):
        ref.set_channel(1, rhs)
        it, rel, ms = ref.solve(1000, 1e-6, 1, 10, 1, w.pure_neumann)
        ref_ms.append(ms)
        ref.set_channel(1, rhs)
        dit, drel, dms = ref.solve_dropin(1000, 1e-6, 1, 10, 1, w.pure_neumann)
        drop_ms.append(dms)
        assert dit == it and abs(drel - rel) <= 1e-12 * rel  # FP64 sums in another order; x and r bitwise below
    print(f"ring512 at the call site: reference {np.median(ref_ms[1:]):.2f} ms per solve; drop-in first call (bind) "
          f"{drop_ms[0]:.2f} ms, later calls median {np.median(drop_ms[1:]):.2f} ms "
          f"({np.median(ref_ms[1:]) / np.median(drop_ms[1:]):.2f}x)")
    O.ref_dropin_lib().refdrop_release_all()
    assert np.median(drop_ms[1:]) < np.median(ref_ms[1:])


@pytest.mark.parametrize("name", ["sphere64_small", "ring512"])
def test_amg_dropin_in_reference_grid(name, built_cache, ref_ok):
    """The drop-in's AMGSolver on the reference's own grid (fresh object per call:
    prepareTypesAndCoeffs, then solve) gives the product's AMGSolver iterations and pressure bit for
    bit on the same right-hand side; after the cell types change, a solve without a new
    preparation is refused (the bound pool was rebuilt), and a prepared one matches again."""
    from cirrus_b200 import AMGSolver, DeviceGrid

    b = built_cache(name)
    w = b.workload
    ref = _ref_grid(b)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    rhs = ref.rhs(b.velocity)
    ref.set_channel(1, rhs)
    ref.set_channel(0, np.zeros_like(rhs))
    got = ref.amg_solve_dropin(True, 1000, 1e-6, 1, 10, 1, w.pure_neumann)
    assert got is not None
    g = DeviceGrid(b.topology)
    g.set_channel(1, rhs)
    s = AMGSolver()
    s.prepare_types_and_coeffs(g)
    it, rel = s.solve(g, is_pure_neumann=w.pure_neumann)
    print(f"{name}: AMG drop-in {got[0]} iters {got[1]:.3e}; product {it} iters {rel:.3e}")
    assert got[0] == it and abs(got[1] - rel) <= 1e-12 * rel
    assert np.array_equal(bits(ref.get_channel(0))[leaf], bits(g.get_channel(0))[leaf])
    g.close()
    # a block of cells turned NEUMANN: the pool is rebuilt on the next call, which needs a new preparation
    base = W.leaf_cell_types(w, b.tiles, b.nbr6)
    cand = [t for t in np.flatnonzero(leaf) if (base[t].reshape(8, 8, 8)[2:6, 2:6, 2:6] == W.INTERIOR).all()]
    moved = base.copy()
    moved[cand[len(cand) // 2]].reshape(8, 8, 8)[2:6, 2:6, 2:6] = W.NEUMANN
    ref.set_ctypes(moved)
    ref.calc_cell_types()
    rhs2 = ref.rhs(b.velocity)  # the right-hand side of the new cell types
    assert ref.amg_solve_dropin(False, 1000, 1e-6, 1, 10, 1, w.pure_neumann) is None
    ref.set_channel(1, rhs2)
    ref.set_channel(0, np.zeros_like(rhs2))
    got2 = ref.amg_solve_dropin(True, 1000, 1e-6, 1, 10, 1, w.pure_neumann)
    assert got2 is not None and got2[1] < 1e-6
