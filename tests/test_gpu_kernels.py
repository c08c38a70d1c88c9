"""Operator parity on the GPU: every CUDA kernel of the solve against the CPU oracle's FP32
mirror of the reference arithmetic, on the same seeded inputs.  Integer/stencil work is
compared bit for bit; the FP64-accumulated dot within 1e-12 relative."""
from __future__ import annotations

import numpy as np
import pytest

from cirrus_b200 import DeviceGrid, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NAMES = ["uniform32_small", "sphere64_small", "ring64_small", "sphere256"]


def setup(b):
    g = DeviceGrid(b.topology)
    for a in range(3):
        g.set_channel(6 + a, b.velocity[a])
    g.projection_rhs()
    f = O.CpuOracle(b.tiles)
    f.set_ctypes(b.ctypes)
    return g, f


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", NAMES)
def test_rhs_bitwise(name, built_cache):
    b = built_cache(name)
    g, f = setup(b)
    assert np.array_equal(bits(g.get_channel(1)), bits(f.rhs(b.velocity)))


@pytest.mark.parametrize("name", NAMES)
def test_full_laplacian_bitwise(name, built_cache):
    b = built_cache(name)
    g, f = setup(b)
    rhs = g.get_channel(1)
    g.set_channel(2, rhs)
    g.full_negative_laplacian(2, 3)
    f.set_channel_f32(2, rhs)
    f.full_lap(O.CpuOracle.FP32, 2, 3)
    lg = (b.tiles[:, 4] & (W.LEAF | W.GHOST)) != 0
    assert np.array_equal(bits(g.get_channel(3))[lg], bits(f.get_channel_f32(3))[lg])
    assert np.array_equal(bits(g.get_channel(2)), bits(f.get_channel_f32(2)))


def same_level_cases(maxl):
    """(tile_level, subtree_level, launch_tile_types, calc_diag) combinations the reference's
    NegativeLaplacianSameLevel128 is called with, plus mixed-context ones."""
    lg, all3 = W.LEAF | W.GHOST, W.LEAF | W.NONLEAF | W.GHOST
    cases = [(-1, -1, lg, 0), (-1, -1, lg, 1), (-1, -1, all3, 0), (-1, min(2, maxl), all3, 0), (-1, maxl, W.NONLEAF, 1)]
    for l in range(maxl + 1):
        cases += [(l, l, W.LEAF | W.NONLEAF, 0), (l, l, W.LEAF | W.NONLEAF, 1), (l, l, W.GHOST, 0), (l, -1, all3, 1)]
    return cases


@pytest.mark.parametrize("name", NAMES)
def test_laplacian_variants_bitwise(name, built_cache):
    """FullNegativeLaplacian with calc_diag, and NegativeLaplacianSameLevel128 for every tile
    array, subtree level and tile-type filter: computed tiles and untouched tiles bit for bit."""
    b = built_cache(name)
    g, f = setup(b)
    rng = np.random.default_rng(11)
    x = rng.standard_normal((b.n, 512)).astype(np.float32)
    y0 = rng.standard_normal((b.n, 512)).astype(np.float32)
    g.set_channel(2, x)
    g.full_negative_laplacian(2, 3, calc_diag=True)
    f.set_channel_f32(2, x)
    f.full_lap_diag(O.CpuOracle.FP32, 2, 3)
    lg = (b.tiles[:, 4] & (W.LEAF | W.GHOST)) != 0
    assert np.array_equal(bits(g.get_channel(3))[lg], bits(f.get_channel_f32(3))[lg])
    maxl = int(b.tiles[:, 0].max())
    for case in same_level_cases(maxl):
        g.set_channel(2, x)
        g.set_channel(3, y0)
        g.negative_laplacian_same_level(*case[:3], 2, 3, bool(case[3]))
        f.set_channel_f32(2, x)
        f.set_channel_f32(3, y0)
        f.lap_same_level(O.CpuOracle.FP32, *case[:3], 2, 3, bool(case[3]))
        assert np.array_equal(bits(g.get_channel(3)), bits(f.get_channel_f32(3))), case


@pytest.mark.parametrize("name", NAMES)
def test_level_operators_bitwise(name, built_cache):
    """GS colour sweeps, residual+restriction and prolongation on every level."""
    b = built_cache(name)
    g, f = setup(b)
    rng = np.random.default_rng(7)
    x = rng.standard_normal((b.n, 512)).astype(np.float32)
    r = rng.standard_normal((b.n, 512)).astype(np.float32)
    maxl = int(b.tiles[:, 0].max())
    for level in range(maxl + 1):
        for color in (0, 1):
            g.set_channel(4, x); g.set_channel(3, r)
            f.set_channel_f32(4, x); f.set_channel_f32(3, r)
            g.gauss_seidel_sweep(level, 4, 3, color)
            f.gs_sweep(O.CpuOracle.FP32, level, 4, 3, color)
            assert np.array_equal(bits(g.get_channel(4)), bits(f.get_channel_f32(4))), (level, color)
        if level >= 1:
            g.set_channel(4, x); g.set_channel(3, r)
            f.set_channel_f32(4, x); f.set_channel_f32(3, r)
            g.residual_and_restrict(level, 4, 3, 3)
            f.residual_restrict(O.CpuOracle.FP32, level, 4, 3, 3)
            assert np.array_equal(bits(g.get_channel(3)), bits(f.get_channel_f32(3))), ("restrict", level)
            g.set_channel(4, x)
            f.set_channel_f32(4, x)
            g.prolongate_and_update(level, 4, 4)
            f.prolongate(O.CpuOracle.FP32, level, 4, 4)
            assert np.array_equal(bits(g.get_channel(4)), bits(f.get_channel_f32(4))), ("prolong", level)


@pytest.mark.parametrize("name", NAMES)
def test_vcycle_bitwise(name, built_cache):
    b = built_cache(name)
    g, f = setup(b)
    rhs = g.get_channel(1)
    g.vcycle(4, 1, 3, 1, 10)
    f.set_channel_f32(1, rhs)
    f.vcycle(O.CpuOracle.FP32, 4, 1, 3, 1, 10)
    leaf = (b.tiles[:, 4] & W.LEAF) != 0
    assert np.array_equal(bits(g.get_channel(4))[leaf], bits(f.get_channel_f32(4))[leaf])


@pytest.mark.parametrize("name", NAMES)
def test_dot(name, built_cache):
    b = built_cache(name)
    g, f = setup(b)
    rhs = g.get_channel(1)
    f.set_channel_f32(1, rhs)
    d_gpu = g.dot(1, 1)
    d_cpu = f.dot(O.CpuOracle.FP32, 1, 1)
    assert abs(d_gpu - d_cpu) <= 1e-12 * abs(d_cpu)
