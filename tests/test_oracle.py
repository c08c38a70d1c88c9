"""The CPU oracle pinned against the reference's own outputs (golden fixtures produced by the
reference CUDA build on a B200), plus its own consistency: FP32 mirror vs FP64 restatement."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_npz
from cirrus_b200 import workloads as W
from oracle import oracle as O

SMALL = ["uniform32_small", "sphere64_small", "sphere64_neumann_small", "ring64_small"]


def oracle_for(b):
    f = O.CpuOracle(b.tiles)
    f.set_ctypes(b.ctypes)
    return f


def leaf_mask(b):
    return (b.tiles[:, 4] & W.LEAF) != 0


def rel_l2(a, ref, mask):
    a = a[mask].astype(np.float64)
    r = ref[mask].astype(np.float64)
    return float(np.linalg.norm(a - r) / max(np.linalg.norm(r), 1e-300))


@pytest.mark.parametrize("name", SMALL)
def test_rhs_matches_reference_bitwise(name, built_cache):
    g = golden_npz(name)
    b = built_cache(name)
    rhs = oracle_for(b).rhs(b.velocity)
    # the divergence writes LEAF and GHOST tiles; NONLEAF tiles keep whatever the channel held
    lg = (b.tiles[:, 4] & (W.LEAF | W.GHOST)) != 0
    assert np.array_equal(rhs[lg].view(np.uint32), g["b"][lg].view(np.uint32))


@pytest.mark.parametrize("name", SMALL)
def test_laplacian_matches_reference(name, built_cache):
    """FullNegativeLaplacian of b: bit-exact with the reference build."""
    g = golden_npz(name)
    b = built_cache(name)
    f = oracle_for(b)
    f.set_channel_f32(2, g["b"])
    f.full_lap(O.CpuOracle.FP32, 2, 3)
    ap = f.get_channel_f32(3)
    lg = (b.tiles[:, 4] & (W.LEAF | W.GHOST)) != 0
    assert np.array_equal(ap[lg].view(np.uint32), g["ap"][lg].view(np.uint32))


@pytest.mark.parametrize("name", SMALL)
def test_vcycle_matches_reference(name, built_cache):
    g = golden_npz(name)
    b = built_cache(name)
    f = oracle_for(b)
    f.set_channel_f32(1, g["b"])
    f.vcycle(O.CpuOracle.FP32, 4, 1, 3, 1, 10)
    z = f.get_channel_f32(4)
    m = leaf_mask(b)
    assert rel_l2(z, g["z"], m) <= 1e-6


@pytest.mark.parametrize("name", SMALL)
def test_solve_matches_reference(name, built_cache):
    g = golden_npz(name)
    b = built_cache(name)
    f = oracle_for(b)
    f.set_channel_f32(1, g["b"])
    it, rel, _ = f.solve(O.CpuOracle.FP32, 1000, 1e-6, 1, 10, 1, b.workload.pure_neumann)
    assert abs(it - int(g["iters"])) <= 1
    assert rel < 1e-6
    x = f.get_channel_f32(0)
    assert rel_l2(x, g["x"], leaf_mask(b)) <= 1e-5


@pytest.mark.parametrize("name", ["uniform32_small", "sphere64_small", "ring64_small"])
def test_fp32_mirror_against_fp64(name, built_cache):
    """The FP32 mirror converges like the FP64 restatement; its pressure error is stated."""
    b = built_cache(name)
    f = oracle_for(b)
    rhs = f.rhs(b.velocity)
    f.set_channel_f32(1, rhs)
    it32, rel32, hist = f.solve(O.CpuOracle.FP32, 1000, 1e-6)
    x32 = f.get_channel_f32(0)
    f.set_channel(O.CpuOracle.FP64, 1, rhs.astype(np.float64))
    it64, rel64, _ = f.solve(O.CpuOracle.FP64, 1000, 1e-10)
    x64 = f.get_channel(O.CpuOracle.FP64, 0)
    assert rel32 < 1e-6 and rel64 < 1e-10
    assert np.all(np.diff(hist) < 0.5 * hist[:-1] + 1e-12) or len(hist) < 3
    err = rel_l2(x32, x64, leaf_mask(b))
    assert err < 1e-4, err


def test_zero_rhs_returns_immediately(built_cache):
    b = built_cache("uniform32_small")
    f = oracle_for(b)
    f.set_channel_f32(1, np.zeros((b.n, 512), np.float32))
    it, rel, _ = f.solve(O.CpuOracle.FP32)
    assert it == 0 and rel == 0.0


def test_pure_neumann_converges(built_cache):
    b = built_cache("sphere64_neumann_small")
    f = oracle_for(b)
    f.set_channel_f32(1, f.rhs(b.velocity))
    it, rel, _ = f.solve(O.CpuOracle.FP32, 1000, 1e-6, pure_neumann=True)
    assert rel < 1e-6 and it < 200


@pytest.mark.parametrize("name", ["uniform32_small", "sphere64_small", "ring64_small"])
def test_damped_jacobi_restatement(name, built_cache):
    """GMGSolver::dampedJacobiSolve restated: the FP32 mirror follows the FP64 restatement, the
    residual falls, a tolerance reached early stops the loop, a zero b gives the reference's 0/0."""
    b = built_cache(name)
    f = oracle_for(b)
    rhs = f.rhs(b.velocity)
    omega = float(np.float32(2.0 / 3.0))
    f.set_channel_f32(1, rhs)
    it10, rel10 = f.damped_jacobi(O.CpuOracle.FP32, 10, 1e-9, omega)
    it40, rel40 = f.damped_jacobi(O.CpuOracle.FP32, 40, 1e-9, omega)
    assert (it10, it40) == (10, 40)
    assert 0.0 < rel40 < rel10 < 1.0
    f.set_channel(O.CpuOracle.FP64, 1, rhs.astype(np.float64))
    it64, rel64 = f.damped_jacobi(O.CpuOracle.FP64, 40, 1e-9, omega)
    assert it64 == 40 and abs(rel64 - rel40) <= 1e-4 * rel64
    # the loop ends at the first residual under tolerance * ||b||: x after 9 updates here
    it, rel = f.damped_jacobi(O.CpuOracle.FP32, 100, rel10 * (1 + 1e-9), omega)
    assert it <= 9 and rel <= rel10 * (1 + 1e-9)
    f.set_channel_f32(1, np.zeros((b.n, 512), np.float32))
    it, rel = f.damped_jacobi(O.CpuOracle.FP32, 10, 1e-6, omega)
    assert it == 0 and np.isnan(rel)


@pytest.mark.parametrize("name", ["sphere64_small", "ring64_small"])
def test_same_level_laplacian_restatement(name, built_cache):
    """NegativeLaplacianSameLevel128 restated, tied to the pinned FullNegativeLaplacian: on x with
    GHOST values already propagated, the same-level operator over all tiles, subtree -1, LEAF|GHOST
    gives FullNegativeLaplacian's result on every tile that receives no GHOST sums; other tiles
    and filters leave the target untouched; the diagonal variant is positive on INTERIOR cells."""
    b = built_cache(name)
    f = oracle_for(b)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((b.n, 512)).astype(np.float32)
    f.set_channel_f32(2, x)
    f.full_lap(O.CpuOracle.FP32, 2, 3)  # also propagates x to the GHOST tiles of channel 2
    full = f.get_channel_f32(3)
    y0 = rng.standard_normal((b.n, 512)).astype(np.float32)
    f.set_channel_f32(4, y0)
    f.lap_same_level(O.CpuOracle.FP32, -1, -1, W.LEAF | W.GHOST, 2, 4)
    same = f.get_channel_f32(4)
    typ, lvl = b.tiles[:, 4], b.tiles[:, 0]
    lg = (typ & (W.LEAF | W.GHOST)) != 0
    coords = {tuple(int(v) for v in r[:4]): i for i, r in enumerate(b.tiles)}
    gparent = np.zeros(b.n, bool)
    for r in b.tiles[(typ & W.GHOST) != 0]:
        p = coords.get((int(r[0]) - 1, int(r[1]) // 2, int(r[2]) // 2, int(r[3]) // 2))
        if p is not None:
            gparent[p] = True
    keep = lg & ~gparent
    assert keep.any() and np.array_equal(same[keep].view(np.uint32), full[keep].view(np.uint32))
    assert np.array_equal(same[~lg].view(np.uint32), y0[~lg].view(np.uint32))
    for l in range(int(lvl.max()) + 1):
        f.set_channel_f32(4, y0)
        f.lap_same_level(O.CpuOracle.FP32, l, l, W.GHOST, 2, 4)
        out = f.get_channel_f32(4)
        untouched = ~((lvl == l) & ((typ & W.GHOST) != 0))
        assert np.array_equal(out[untouched].view(np.uint32), y0[untouched].view(np.uint32))
    f.set_channel_f32(4, y0)
    f.lap_same_level(O.CpuOracle.FP32, -1, -1, W.LEAF, 2, 4, diag=True)
    d = f.get_channel_f32(4)
    leaf = (typ & W.LEAF) != 0
    interior = (b.ctypes & W.INTERIOR) != 0
    assert np.all(d[leaf][interior[leaf]] > 0)
