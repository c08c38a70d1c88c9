"""Synthetic Poisson workloads with the shapes of the benchmark configurations.

Each workload fixes: the root tiles, per-level refinement masks (the level-target function of
IterativeRefine, src/PoissonGrid.h:316-326), the leaf cell-type rule, and a seeded face-velocity
field whose discrete divergence is the right-hand side.  There are no datasets: every input is
generated from a seed.

Cell-type rule (restating FluidParams::cellType, src/FluidParams.cu:125-144 and :241-244):
a LEAF cell with a missing same-level neighbour tile is NEUMANN, except that a missing +z
neighbour alone makes it DIRICHLET (an open top, p = 0) unless the workload is pure Neumann;
otherwise a cell whose centre lies inside the obstacle is NEUMANN; else INTERIOR.

Velocity: i.i.d. N(0,1) on the three lower faces of every cell, from a counter-based generator
keyed by (seed, level, global cell, axis) so that every consumer regenerates identical values.

Workloads:
  uniform128   uniform 128^3 grid (level-4 leaves, 16^3 tiles), Neumann walls, Dirichlet top
  sphere256    leaves at levels 3-5, level 5 within 8 fine cells of the sphere |x-(.5,.5,.5)|=.2,
               solid sphere NEUMANN; also a pure-Neumann variant (no open top)
  ring512      domain 1x1x2 (roots (0,0,0),(0,0,1)), leaves at levels 2-6, level 6 where the
               vorticity of a Gaussian-core vortex ring (R=.15, core .02, centre (.5,.5,.25),
               axis +z) exceeds 10% of its maximum; box obstacle centre (.5,.5,1.0), half-extent .1
Small variants (`*_small`) keep the same rules at sizes the CPU oracle solves in seconds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

LEAF, NONLEAF, GHOST = 1, 2, 4
DIRICHLET, INTERIOR, NEUMANN = 1, 2, 4
FLUID_EULER_LOG2_HASH = (16, 16, 16, 16, 16, 16, 18, 16, 16, 16)


@dataclass
class Workload:
    name: str
    roots: list[tuple[int, int, int]]
    root_extent: tuple[int, int, int]               # level-0 tiles per axis
    masks: list[np.ndarray | None]                   # per level: refine LEAF tile at level l
    pure_neumann: bool = False
    obstacle: Callable[[np.ndarray], np.ndarray] | None = None  # (N,3) centres -> bool inside
    seed: int = 0
    h0: float = 1.0 / 8
    log2_hash: tuple[int, ...] = FLUID_EULER_LOG2_HASH
    description: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def num_layers(self) -> int:
        return len(self.log2_hash)

    def mask_dims(self) -> np.ndarray:
        dims = np.zeros((self.num_layers, 3), dtype=np.int32)
        for l, m in enumerate(self.masks):
            if m is not None:
                dims[l] = m.shape
        return dims


# ----------------------------------------------------------------------------- geometry
def _tile_boxes(level: int, extent: tuple[int, int, int], h0: float):
    """Lower/upper corners of all tiles of a level (tile width 8*h0/2^level), shape (nx,ny,nz,3)."""
    n = [e << level for e in extent]
    w = 8 * h0 / (1 << level)
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), axis=-1).astype(np.float64)
    return idx * w, (idx + 1) * w


def _box_point_dist2(lo: np.ndarray, hi: np.ndarray, p: np.ndarray) -> np.ndarray:
    d = np.maximum(np.maximum(lo - p, 0.0), p - hi)
    return (d * d).sum(axis=-1)


def _box_far_dist2(lo: np.ndarray, hi: np.ndarray, p: np.ndarray) -> np.ndarray:
    d = np.maximum(np.abs(lo - p), np.abs(hi - p))
    return (d * d).sum(axis=-1)


def sphere_band_masks(base: int, fine: int, center, radius: float, band: float, extent=(1, 1, 1), h0=1 / 8, num_layers=10):
    """Refine every tile below `base`; refine tiles within `band` of the sphere surface below `fine`."""
    c = np.asarray(center, dtype=np.float64)
    masks: list[np.ndarray | None] = [None] * num_layers
    for l in range(fine):
        lo, hi = _tile_boxes(l, extent, h0)
        if l < base:
            masks[l] = np.ones(lo.shape[:3], dtype=np.uint8)
            continue
        dmin2 = _box_point_dist2(lo, hi, c)
        dmax2 = _box_far_dist2(lo, hi, c)
        near = (dmin2 <= (radius + band) ** 2) & (dmax2 >= max(radius - band, 0.0) ** 2)
        masks[l] = near.astype(np.uint8)
    return masks


def ring_masks(base: int, fine: int, center, major: float, core: float, frac: float, extent=(1, 1, 2), h0=1 / 8,
               num_layers=10, samples: int = 2048):
    """Refine tiles below `base`; below `fine`, refine tiles whose box comes within the radius
    where |omega| of a Gaussian-core ring falls to `frac` of its maximum
    (|omega| ~ exp(-s^2/core^2), s = distance to the core circle)."""
    c = np.asarray(center, dtype=np.float64)
    s_thr = core * math.sqrt(math.log(1.0 / frac))
    th = 2 * np.pi * np.arange(samples) / samples
    pts = np.stack([c[0] + major * np.cos(th), c[1] + major * np.sin(th), np.full_like(th, c[2])], axis=-1)
    masks: list[np.ndarray | None] = [None] * num_layers
    for l in range(fine):
        lo, hi = _tile_boxes(l, extent, h0)
        if l < base:
            masks[l] = np.ones(lo.shape[:3], dtype=np.uint8)
            continue
        shape = lo.shape[:3]
        lo2, hi2 = lo.reshape(-1, 3), hi.reshape(-1, 3)
        # cheap prefilter against the ring's bounding box
        rlo = c - np.array([major + s_thr, major + s_thr, s_thr])
        rhi = c + np.array([major + s_thr, major + s_thr, s_thr])
        cand = np.all((hi2 >= rlo) & (lo2 <= rhi), axis=1)
        near = np.zeros(lo2.shape[0], dtype=bool)
        ids = np.nonzero(cand)[0]
        for start in range(0, ids.size, 4096):
            sl = ids[start:start + 4096]
            d2 = _box_point_dist2(lo2[sl, None, :], hi2[sl, None, :], pts[None, :, :]).min(axis=1)
            near[sl] = d2 <= s_thr * s_thr
        masks[l] = near.reshape(shape).astype(np.uint8)
    return masks


def sphere_obstacle(center, radius):
    c = np.asarray(center, dtype=np.float64)
    r2 = radius * radius

    def inside(p: np.ndarray) -> np.ndarray:
        d = p - c
        return (d * d).sum(axis=-1) <= r2
    return inside


def box_obstacle(center, half):
    c = np.asarray(center, dtype=np.float64)

    def inside(p: np.ndarray) -> np.ndarray:
        return np.all(np.abs(p - c) <= half, axis=-1)
    return inside


# ----------------------------------------------------------------------------- workloads
def uniform(level: int = 4, seed: int = 0) -> Workload:
    masks: list[np.ndarray | None] = [None] * 10
    for l in range(level):
        masks[l] = np.ones((1 << l,) * 3, dtype=np.uint8)
    n = 8 << level
    return Workload(name=f"uniform{n}", roots=[(0, 0, 0)], root_extent=(1, 1, 1), masks=masks, seed=seed,
                    description=f"uniform {n}^3, Neumann walls, Dirichlet top")


def sphere(base: int = 3, fine: int = 5, seed: int = 0, pure_neumann: bool = False, band_cells: int = 8) -> Workload:
    band = band_cells / float(8 << fine)
    masks = sphere_band_masks(base, fine, (0.5, 0.5, 0.5), 0.2, band)
    eff = 8 << fine
    return Workload(name=f"sphere{eff}" + ("_neumann" if pure_neumann else ""), roots=[(0, 0, 0)], root_extent=(1, 1, 1),
                    masks=masks, pure_neumann=pure_neumann, obstacle=sphere_obstacle((0.5, 0.5, 0.5), 0.2), seed=seed,
                    description=f"leaves at levels {base}-{fine}, sphere r=0.2 band {band_cells} fine cells")


def ring(base: int = 2, fine: int = 6, seed: int = 0) -> Workload:
    masks = ring_masks(base, fine, (0.5, 0.5, 0.25), 0.15, 0.02, 0.1)
    eff = 8 << fine
    return Workload(name=f"ring{eff}", roots=[(0, 0, 0), (0, 0, 1)], root_extent=(1, 1, 2), masks=masks,
                    obstacle=box_obstacle((0.5, 0.5, 1.0), 0.1), seed=seed,
                    description=f"domain 1x1x2, leaves at levels {base}-{fine}, vortex ring R=.15 core .02 >10% |w|, "
                                f"box obstacle c=(.5,.5,1) half .1")


def random_spheres(seed: int = 0) -> Workload:
    """One instance of the batched configuration: effective size log-uniform over 64^3, 128^3,
    256^3 (finest level 3-5), 1-4 levels of leaves, refinement in an 8-fine-cell band around 1-5
    seeded spheres of radius U(0.05, 0.25); Neumann box walls with a Dirichlet top."""
    rng = np.random.default_rng(0x5EED0000 + seed)
    fine = int(rng.integers(3, 6))
    depth = int(rng.integers(1, 5))
    base = max(fine - depth + 1, 0)
    k = int(rng.integers(1, 6))
    centers = rng.uniform(0.2, 0.8, size=(k, 3))
    radii = rng.uniform(0.05, 0.25, size=k)
    band = 8 / float(8 << fine)
    masks: list[np.ndarray | None] = [None] * 10
    for l in range(fine):
        lo, hi = _tile_boxes(l, (1, 1, 1), 1 / 8)
        if l < base:
            masks[l] = np.ones(lo.shape[:3], dtype=np.uint8)
            continue
        near = np.zeros(lo.shape[:3], dtype=bool)
        for c, r in zip(centers, radii):
            dmin2 = _box_point_dist2(lo, hi, c)
            dmax2 = _box_far_dist2(lo, hi, c)
            near |= (dmin2 <= (r + band) ** 2) & (dmax2 >= max(r - band, 0.0) ** 2)
        masks[l] = near.astype(np.uint8)
    eff = 8 << fine
    return Workload(name=f"spheres{eff}_d{depth}_s{seed}", roots=[(0, 0, 0)], root_extent=(1, 1, 1), masks=masks, seed=seed,
                    description=f"{eff}^3 effective, leaves at levels {base}-{fine}, {k} random spheres",
                    meta={"fine": fine, "depth": depth, "spheres": k, "velocity": "stream"})


def random_session(seed: int = 0) -> Workload:
    """One problem of the serving configuration: effective size log-uniform over 32^3 - 512^3
    (finest level 2-6, the exponent drawn uniformly), 1-5 levels of leaves, refinement around a
    seeded sphere (band of 8 fine cells) or a seeded vortex ring (the ring's 10%-vorticity tube);
    Neumann box walls with a Dirichlet top, unit cube.  The number of levels is at least fine - 3,
    so no level is refined uniformly beyond 128^3 (keeps every session within a few GB)."""
    rng = np.random.default_rng(0xC5C50000 + seed)
    fine = int(np.floor(rng.uniform(2.0, 7.0)))  # 8 << fine effective cells: 32 ... 512, log-uniform
    depth = int(rng.integers(max(1, fine - 3), min(5, fine + 1) + 1))
    base = fine - depth + 1
    kind = "sphere" if rng.random() < 0.5 else "ring"
    eff = 8 << fine
    if kind == "sphere":
        c = rng.uniform(0.3, 0.7, size=3)
        r = float(rng.uniform(0.1, 0.25))
        band = 8 / float(eff)
        masks: list[np.ndarray | None] = [None] * 10
        for l in range(fine):
            lo, hi = _tile_boxes(l, (1, 1, 1), 1 / 8)
            if l < base:
                masks[l] = np.ones(lo.shape[:3], dtype=np.uint8)
                continue
            dmin2 = _box_point_dist2(lo, hi, c)
            dmax2 = _box_far_dist2(lo, hi, c)
            masks[l] = ((dmin2 <= (r + band) ** 2) & (dmax2 >= max(r - band, 0.0) ** 2)).astype(np.uint8)
        obstacle = sphere_obstacle(c, r)
        desc = f"sphere c={np.round(c, 3).tolist()} r={r:.3f}"
    else:
        c = (float(rng.uniform(0.35, 0.65)), float(rng.uniform(0.35, 0.65)), float(rng.uniform(0.3, 0.7)))
        major = float(rng.uniform(0.1, 0.2))
        masks = ring_masks(base, fine, c, major, 0.02, 0.1, extent=(1, 1, 1))
        obstacle = None
        desc = f"vortex ring c={np.round(c, 3).tolist()} R={major:.3f}"
    return Workload(name=f"session{eff}_d{depth}_{kind}_s{seed}", roots=[(0, 0, 0)], root_extent=(1, 1, 1), masks=masks,
                    obstacle=obstacle, seed=seed, description=f"{eff}^3 effective, leaves at levels {base}-{fine}, {desc}",
                    meta={"fine": fine, "depth": depth, "kind": kind, "velocity": "stream"})


def serving_sessions(count: int = 16, seed0: int = 0) -> list[Workload]:
    """The serving configuration's problems: `count` independent random_session instances."""
    return [random_session(seed0 + i) for i in range(count)]


def stream_velocity(tiles: np.ndarray, seed: int) -> np.ndarray:
    """(3, n, 512) float32 N(0,1) lower-face velocities on LEAF tiles from one seeded stream in
    all-tiles order (reproducible for a given tile list; faster than face_velocity)."""
    n = tiles.shape[0]
    out = np.zeros((3, n, 512), dtype=np.float32)
    leaf = np.flatnonzero((tiles[:, 4] & LEAF) != 0)
    rng = np.random.default_rng(0xF00D0000 + seed)
    out[:, leaf] = rng.standard_normal((3, leaf.size, 512), dtype=np.float32)
    return out


def batch_of_spheres(count: int = 64, seed0: int = 0) -> list[Workload]:
    """The batched configuration: `count` independent random_spheres instances."""
    return [random_spheres(seed0 + i) for i in range(count)]


WORKLOADS: dict[str, Callable[..., Workload]] = {
    "uniform128": lambda seed=0: uniform(4, seed),
    "sphere256": lambda seed=0: sphere(3, 5, seed),
    "sphere256_neumann": lambda seed=0: sphere(3, 5, seed, pure_neumann=True),
    "ring512": lambda seed=0: ring(2, 6, seed),
    # CPU-oracle sizes
    "uniform32_small": lambda seed=0: uniform(2, seed),
    "sphere64_small": lambda seed=0: sphere(1, 3, seed, band_cells=6),
    "sphere64_neumann_small": lambda seed=0: sphere(1, 3, seed, pure_neumann=True, band_cells=6),
    "ring64_small": lambda seed=0: ring(1, 3, seed),
}


def make(name: str, seed: int = 0) -> Workload:
    return WORKLOADS[name](seed=seed)


# ----------------------------------------------------------------------------- cell types
def cell_centers(tiles: np.ndarray, h0: float = 1 / 8) -> np.ndarray:
    """(n, 512, 3) cell centres in world coordinates."""
    o = np.arange(512)
    loc = np.stack([o >> 6, (o >> 3) & 7, o & 7], axis=-1)
    g = tiles[:, None, 1:4].astype(np.int64) * 8 + loc[None]
    h = h0 / (1 << tiles[:, 0].astype(np.int64))
    return (g + 0.5) * h[:, None, None]


def leaf_cell_types(w: Workload, tiles: np.ndarray, nbr6: np.ndarray) -> np.ndarray:
    """Cell types of LEAF tiles (other tiles left 0, filled by CalcCellTypesFromLeafs)."""
    n = tiles.shape[0]
    ct = np.zeros((n, 8, 8, 8), dtype=np.uint8)
    leaf = (tiles[:, 4] & LEAF) != 0
    neu = np.zeros((n, 8, 8, 8), dtype=bool)
    dir_ = np.zeros((n, 8, 8, 8), dtype=bool)
    # same-level neighbour voxel missing <=> the cell is on a tile face whose neighbour tile is absent
    for axis in range(3):
        for sgn, col in ((-1, axis), (1, axis + 3)):
            missing = nbr6[:, col] < 0
            sl = [slice(None)] * 4
            sl[axis + 1] = 0 if sgn < 0 else 7
            face = np.zeros((n, 8, 8, 8), dtype=bool)
            face[tuple(sl)] = True
            hit = face & missing[:, None, None, None]
            if axis == 2 and sgn == 1 and not w.pure_neumann:
                dir_ |= hit
            else:
                neu |= hit
    t = np.full((n, 8, 8, 8), INTERIOR, dtype=np.uint8)
    if w.obstacle is not None:
        inside = w.obstacle(cell_centers(tiles, w.h0).reshape(-1, 3)).reshape(n, 8, 8, 8)
        t[inside] = NEUMANN
    t[dir_] = DIRICHLET
    t[neu] = NEUMANN
    ct[leaf] = t[leaf]
    return ct.reshape(n, 512)


# ----------------------------------------------------------------------------- velocity
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = x
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def face_velocity(tiles: np.ndarray, seed: int) -> np.ndarray:
    """(3, n, 512) float32 N(0,1) lower-face velocities on LEAF tiles (0 elsewhere); the value of
    a face depends only on (seed, level, global cell, axis)."""
    n = tiles.shape[0]
    out = np.zeros((3, n, 512), dtype=np.float32)
    leaf = np.flatnonzero((tiles[:, 4] & LEAF) != 0)
    m = leaf.size
    if m == 0:
        return out
    o = np.arange(512)
    loc = np.stack([o >> 6, (o >> 3) & 7, o & 7], axis=-1).astype(np.int64)
    g = tiles[leaf, None, 1:4].astype(np.int64) * 8 + loc[None]
    lev = np.broadcast_to(tiles[leaf, None, 0].astype(np.int64), (m, 512))
    for axis in range(3):
        k = _splitmix(np.full((m, 512), np.uint64(seed), dtype=np.uint64))
        for comp in (lev, g[..., 0], g[..., 1], g[..., 2], np.full((m, 512), axis, dtype=np.int64)):
            k = _splitmix(k ^ comp.astype(np.uint64))
        u1 = ((_splitmix(k) >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
        u2 = ((_splitmix(k ^ np.uint64(0x5851F42D4C957F2D)) >> np.uint64(11)).astype(np.float64)) * (1.0 / 9007199254740992.0)
        z = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
        out[axis, leaf] = z.astype(np.float32)
    return out


# ----------------------------------------------------------------------------- assembly
@dataclass
class Built:
    """A workload turned into the arrays every consumer takes (all-tiles order)."""
    workload: Workload
    tiles: np.ndarray          # (n, 5) level, x, y, z, type
    nbr6: np.ndarray           # (n, 6) x-, y-, z-, x+, y+, z+
    ctypes: np.ndarray         # (n, 512) after CalcCellTypesFromLeafs
    velocity: np.ndarray       # (3, n, 512)
    topology: object = None    # the product Topology (keeps handles alive)

    @property
    def n(self) -> int:
        return self.tiles.shape[0]

    def dof(self) -> int:
        leaf = (self.tiles[:, 4] & LEAF) != 0
        return int(((self.ctypes[leaf] & INTERIOR) != 0).sum())

    def counts(self) -> dict:
        t = self.tiles
        out = {"tiles": int(t.shape[0]), "dof": self.dof(), "max_level": int(t[:, 0].max())}
        for name, bit in (("leaf", LEAF), ("nonleaf", NONLEAF), ("ghost", GHOST)):
            out[name] = int(((t[:, 4] & bit) != 0).sum())
        return out


def build(w: Workload):
    """Build the topology with the product library (host builder), apply the cell-type rule,
    run CalcCellTypesFromLeafs and generate the face velocity."""
    from . import Topology

    topo = Topology(w.h0, w.log2_hash)
    for r in w.roots:
        topo.set_tile(0, r, LEAF)
    topo.compress()
    topo.spawn_ghost_tiles()
    topo.iterative_refine(masks=w.masks)
    tiles = topo.tiles()
    nbr6 = topo.neighbor_tiles()
    topo.set_cell_types(leaf_cell_types(w, tiles, nbr6))
    topo.calc_cell_types_from_leafs()
    ct = topo.cell_types()
    vel = stream_velocity(tiles, w.seed) if w.meta.get("velocity") == "stream" else face_velocity(tiles, w.seed)
    return Built(w, tiles, nbr6, ct, vel, topo)
