"""cirrus_b200 -- B200-native GMG-PCG pressure solver for adaptive octree-tile grids.

Python host layer over the C ABI of include/cirrus_b200.h.  It mirrors the reference's
interface for the Poisson path (wang-mengdi/Cirrus):

  reference                                   here
  HADeviceGrid(h0, log2 hashes) + setTileHost  Topology(...).set_tile(...)
  compressHost / syncHostAndDevice             Topology.compress()
  SpawnGhostTiles / IterativeRefine            Topology.spawn_ghost_tiles() / iterative_refine()
  CalcCellTypesFromLeafs                       Topology.calc_cell_types_from_leafs()
  tile channels on the device                  DeviceGrid (HBM tile pool)
  FullNegativeLaplacian, VCycle, Dot, ...      DeviceGrid methods
  GMGSolver(one_over_alpha, prolong_coeff)     GMGSolver(...)
    .solve(grid, verbose, max_iters, tol,       .solve(grid, verbose, max_iters, tol,
           level_iters, coarsest_iters,                level_iters, coarsest_iters,
           sync_stride, is_pure_neumann)               sync_stride, is_pure_neumann)
           -> (iters, relative_residual)               -> (iters, relative_residual)

All compute runs in the native library on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Sequence

import numpy as np

from ._native import (CirrusError, Completion, LEVEL_TARGET_FN, SolveParams, SolveResult, check, lib, loaded_lib)

__all__ = [
    "LEAF", "NONLEAF", "GHOST", "DIRICHLET", "INTERIOR", "NEUMANN",
    "X_CHANNEL", "B_CHANNEL", "R_CHANNEL", "P_CHANNEL", "AP_CHANNEL", "Z_CHANNEL", "TMP_CHANNEL", "U_CHANNEL",
    "FLUID_EULER_LOG2_HASH", "Topology", "DeviceTopology", "DeviceGrid", "GMGSolver", "AMGSolver", "Holder", "CirrusError", "lib",
]

LEAF, NONLEAF, GHOST = 1, 2, 4
# kernels of cirrus_bench_launch
KERNEL_LAPLACIAN, KERNEL_GS_SWEEP, KERNEL_PRESMOOTH, KERNEL_PROLONG_SWEEP, KERNEL_RESIDUAL_RESTRICT, KERNEL_COARSE, KERNEL_DOT = range(7)
DIRICHLET, INTERIOR, NEUMANN = 1, 2, 4
X_CHANNEL, B_CHANNEL, R_CHANNEL, P_CHANNEL, AP_CHANNEL, Z_CHANNEL, TMP_CHANNEL, U_CHANNEL = 0, 1, 1, 2, 3, 4, 5, 6
PRECISION_FP32, PRECISION_MIXED_FP64 = 0, 1

# per-level hash sizes of FluidEuler's grid (src/FluidEuler.h:416)
FLUID_EULER_LOG2_HASH = (16, 16, 16, 16, 16, 16, 18, 16, 16, 16)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class Topology:
    """Octree of 8^3 tiles built on the host exactly as the reference builds it."""

    def __init__(self, h0: float = 1.0 / 8, levels_log2_hash: Sequence[int] = FLUID_EULER_LOG2_HASH):
        self.num_layers = len(levels_log2_hash)
        self.h0 = float(h0)
        arr = (C.c_uint32 * self.num_layers)(*levels_log2_hash)
        h = C.c_void_p()
        check(lib().cirrus_topology_create(self.num_layers, arr, self.h0, C.byref(h)), "cirrus_topology_create")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        L = loaded_lib()
        if h is not None and h.value and L is not None:
            L.cirrus_topology_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def set_tile(self, level: int, coord: Sequence[int], tile_type: int = LEAF) -> None:
        x, y, z = (int(c) for c in coord)
        check(lib().cirrus_topology_set_tile(self._h, level, x, y, z, tile_type), "cirrus_topology_set_tile")

    def compress(self) -> None:
        check(lib().cirrus_topology_compress(self._h), "cirrus_topology_compress")

    def spawn_ghost_tiles(self) -> None:
        check(lib().cirrus_topology_spawn_ghost_tiles(self._h), "cirrus_topology_spawn_ghost_tiles")

    def refine_leafs_one_step(self, level_target: Callable[[int, int, int, int], int]) -> list[int]:
        fn = LEVEL_TARGET_FN(lambda _u, l, x, y, z: int(level_target(l, x, y, z)))
        out = (C.c_int * self.num_layers)()
        check(lib().cirrus_topology_refine_leafs_one_step(self._h, fn, None, out), "cirrus_topology_refine_leafs_one_step")
        return list(out)

    def iterative_refine(self, level_target: Callable[[int, int, int, int], int] | None = None,
                         masks: Sequence[np.ndarray | None] | None = None) -> None:
        """IterativeRefine with a level-target callback, or with dense per-level masks
        (masks[l][x, y, z] != 0 -> a LEAF tile at level l is refined)."""
        if masks is not None:
            keep, ptrs, dims = _mask_args(masks, self.num_layers)
            check(lib().cirrus_topology_iterative_refine_masks(self._h, ptrs, dims), "cirrus_topology_iterative_refine_masks")
            del keep
        else:
            fn = LEVEL_TARGET_FN(lambda _u, l, x, y, z: int(level_target(l, x, y, z)))
            check(lib().cirrus_topology_iterative_refine(self._h, fn, None), "cirrus_topology_iterative_refine")

    @property
    def num_tiles(self) -> int:
        n = C.c_int()
        check(lib().cirrus_topology_num_tiles(self._h, C.byref(n)), "cirrus_topology_num_tiles")
        return n.value

    @property
    def max_level(self) -> int:
        n = C.c_int()
        check(lib().cirrus_topology_max_level(self._h, C.byref(n)), "cirrus_topology_max_level")
        return n.value

    def tiles(self) -> np.ndarray:
        """(n, 5) int32: level, x, y, z, type in all-tiles order."""
        out = np.empty((self.num_tiles, 5), dtype=np.int32)
        check(lib().cirrus_topology_tiles(self._h, _ptr(out, C.c_int32)), "cirrus_topology_tiles")
        return out

    def hash_slots(self) -> np.ndarray:
        out = np.empty(self.num_tiles, dtype=np.int32)
        check(lib().cirrus_topology_hash_slots(self._h, _ptr(out, C.c_int32)), "cirrus_topology_hash_slots")
        return out

    def neighbor_tiles(self) -> np.ndarray:
        """(n, 6) int32 (x-, y-, z-, x+, y+, z+) as CalculateNeighborTiles fills mNeighbors."""
        out = np.empty((self.num_tiles, 6), dtype=np.int32)
        check(lib().cirrus_topology_neighbor_tiles(self._h, _ptr(out, C.c_int32)), "cirrus_topology_neighbor_tiles")
        return out

    def set_cell_types(self, ctypes: np.ndarray) -> None:
        a = np.ascontiguousarray(ctypes, dtype=np.uint8).reshape(self.num_tiles, 512)
        check(lib().cirrus_topology_set_cell_types(self._h, _ptr(a, C.c_uint8)), "cirrus_topology_set_cell_types")

    def cell_types(self) -> np.ndarray:
        out = np.empty((self.num_tiles, 512), dtype=np.uint8)
        check(lib().cirrus_topology_cell_types(self._h, _ptr(out, C.c_uint8)), "cirrus_topology_cell_types")
        return out

    def calc_cell_types_from_leafs(self) -> None:
        check(lib().cirrus_topology_calc_cell_types_from_leafs(self._h), "cirrus_topology_calc_cell_types_from_leafs")


def _mask_args(masks, num_layers):
    keep = []
    ptrs = (C.POINTER(C.c_uint8) * num_layers)()
    dims = (C.c_int * (3 * num_layers))()
    for l in range(num_layers):
        m = masks[l] if l < len(masks) else None
        if m is None:
            ptrs[l] = C.POINTER(C.c_uint8)()
            continue
        a = np.ascontiguousarray(m, dtype=np.uint8)
        keep.append(a)
        ptrs[l] = _ptr(a, C.c_uint8)
        dims[3 * l], dims[3 * l + 1], dims[3 * l + 2] = a.shape
    return keep, ptrs, dims


class DeviceGrid:
    """The tile pool of a finalised topology resident on the current CUDA device."""

    def __init__(self, topology: "Topology | Sequence[Topology]"):
        """One instance (a Topology) or a batch of independent instances (a sequence of them) in
        one tile pool; a batch is solved together by GMGSolver.solve_batch."""
        h = C.c_void_p()
        if isinstance(topology, Topology):
            check(lib().cirrus_grid_create(topology.handle, C.byref(h)), "cirrus_grid_create")
            topos = [topology]
        else:
            topos = list(topology)
            arr = (C.c_void_p * len(topos))(*[t.handle.value for t in topos])
            check(lib().cirrus_grid_create_batch(arr, len(topos), C.byref(h)), "cirrus_grid_create_batch")
        self._h = h
        n = C.c_int()
        check(lib().cirrus_grid_num_tiles(h, C.byref(n)), "cirrus_grid_num_tiles")
        self.num_tiles = n.value
        self.num_instances = len(topos)
        self.instance_tiles = [t.num_tiles for t in topos]
        self.tiles = topos[0].tiles() if len(topos) == 1 else None

    @classmethod
    def from_arrays(cls, h0: float, levels_log2_hash: Sequence[int], tiles5: np.ndarray, cell_types: np.ndarray,
                    b: np.ndarray | None = None, x0: np.ndarray | None = None) -> "DeviceGrid":
        """A device grid straight from a reference grid's arrays (cirrus_grid_create_from_desc):
        tiles5 = (n, 5) int32 rows (level, x, y, z, type), level-major in the reference's order;
        cell_types = (n, 512) uint8; optional b and x0 = (n, 512) float32."""
        from ._native import GridDesc

        t5 = np.ascontiguousarray(tiles5, dtype=np.int32)
        n, L = t5.shape[0], len(levels_log2_hash)
        counts = np.bincount(t5[:, 0], minlength=L).astype(np.int32)
        coords = np.ascontiguousarray(t5[:, 1:4])
        types = np.ascontiguousarray(t5[:, 4].astype(np.uint8))
        ct = np.ascontiguousarray(cell_types, dtype=np.uint8)
        log2 = (C.c_uint32 * L)(*levels_log2_hash)
        d = GridDesc()
        d.h0, d.num_layers, d.log2_hash = float(h0), L, log2
        d.tiles_per_level = _ptr(counts, C.c_int32)
        d.coords = _ptr(coords, C.c_int32)
        d.types = _ptr(types, C.c_uint8)
        d.cell_types = _ptr(ct, C.c_uint8)
        keep = []
        for name, arr in (("b", b), ("x0", x0)):
            if arr is not None:
                a = np.ascontiguousarray(arr, dtype=np.float32)
                keep.append(a)
                setattr(d, name, _ptr(a, C.c_float))
        h = C.c_void_p()
        check(lib().cirrus_grid_create_from_desc(C.byref(d), C.byref(h)), "cirrus_grid_create_from_desc")
        self = cls.__new__(cls)
        self._h = h
        self.num_tiles = n
        self.num_instances = 1
        self.instance_tiles = [n]
        self.tiles = t5
        return self

    def __del__(self):
        h = getattr(self, "_h", None)
        L = loaded_lib()
        if h is not None and h.value and L is not None:
            L.cirrus_grid_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    @property
    def handle(self):
        return self._h

    @property
    def dof(self) -> int:
        d = C.c_int64()
        check(lib().cirrus_grid_dof(self._h, C.byref(d)), "cirrus_grid_dof")
        return d.value

    @property
    def device_bytes(self) -> int:
        d = C.c_size_t()
        check(lib().cirrus_grid_device_bytes(self._h, C.byref(d)), "cirrus_grid_device_bytes")
        return d.value

    def set_channel(self, channel: int, values: np.ndarray, stream: int = 0) -> None:
        a = np.ascontiguousarray(values, dtype=np.float32).reshape(self.num_tiles * 512)
        check(lib().cirrus_grid_set_channel(self._h, channel, _ptr(a, C.c_float), C.c_void_p(stream)), "cirrus_grid_set_channel")

    def get_channel(self, channel: int, stream: int = 0) -> np.ndarray:
        out = np.empty((self.num_tiles, 512), dtype=np.float32)
        check(lib().cirrus_grid_get_channel(self._h, channel, _ptr(out, C.c_float), C.c_void_p(stream)), "cirrus_grid_get_channel")
        return out

    def set_channel_instance(self, instance: int, channel: int, values: np.ndarray, stream: int = 0) -> None:
        a = np.ascontiguousarray(values, dtype=np.float32).reshape(self.instance_tiles[instance] * 512)
        check(lib().cirrus_grid_set_channel_instance(self._h, instance, channel, _ptr(a, C.c_float), C.c_void_p(stream)),
              "cirrus_grid_set_channel_instance")

    def get_channel_instance(self, instance: int, channel: int, stream: int = 0) -> np.ndarray:
        out = np.empty((self.instance_tiles[instance], 512), dtype=np.float32)
        check(lib().cirrus_grid_get_channel_instance(self._h, instance, channel, _ptr(out, C.c_float), C.c_void_p(stream)),
              "cirrus_grid_get_channel_instance")
        return out

    def autotune(self, reps: int = 20, stream: int = 0) -> None:
        """Pick the fastest launch shape of each staged stencil kernel per level on this grid
        (results are unchanged by the choice); overwrites channels 2-5."""
        check(lib().cirrus_grid_autotune(self._h, reps, C.c_void_p(stream)), "cirrus_grid_autotune")

    def set_launch_shape(self, shape: int, kernel: int = -1, level: int = -1) -> None:
        """Set the launch shape (0..7) of one staged stencil kernel (KERNEL_*, -1: all) on one
        level (-1: all); results are unchanged by the choice."""
        check(lib().cirrus_grid_set_launch_shape(self._h, kernel, level, shape), "cirrus_grid_set_launch_shape")

    def get_launch_shape(self, kernel: int, level: int = 0) -> int:
        v = C.c_int(0)
        check(lib().cirrus_grid_get_launch_shape(self._h, kernel, level, C.byref(v)), "cirrus_grid_get_launch_shape")
        return v.value

    def set_launch_mode(self, direct: bool) -> None:
        """direct=False (default): each solve is one CUDA graph launch; direct=True: the same
        kernels launched one by one from the host (visible to launch tracers).  Same bits."""
        check(lib().cirrus_grid_set_launch_mode(self._h, 1 if direct else 0), "cirrus_grid_set_launch_mode")

    def bench_launch(self, kernel: int, level: int = 0, reps: int = 1, stream: int = 0) -> None:
        """Launch one solve kernel `reps` times on `stream` (for timing with the caller's events);
        overwrites channels 2-5."""
        check(lib().cirrus_bench_launch(self._h, kernel, level, reps, C.c_void_p(stream)), "cirrus_bench_launch")

    def instance_dof(self, instance: int) -> int:
        d = C.c_int64()
        check(lib().cirrus_grid_instance_info(self._h, instance, None, C.byref(d)), "cirrus_grid_instance_info")
        return d.value

    def copy_channel(self, dst_channel: int, src_channel: int, stream: int = 0) -> None:
        check(lib().cirrus_grid_copy_channel(self._h, dst_channel, src_channel, C.c_void_p(stream)), "cirrus_grid_copy_channel")

    def channel_ptr(self, channel: int) -> int:
        p = C.c_void_p()
        check(lib().cirrus_grid_channel_ptr(self._h, channel, C.byref(p)), "cirrus_grid_channel_ptr")
        return p.value

    # operators ------------------------------------------------------------------------
    def full_negative_laplacian(self, x_channel: int, Ax_channel: int, calc_diag: bool = False, stream: int = 0) -> None:
        """FullNegativeLaplacian(grid, x_channel, Ax_channel, calc_diag) (src/GMGSolver.cu:203-213)."""
        check(lib().cirrus_full_negative_laplacian_ex(self._h, x_channel, Ax_channel, int(bool(calc_diag)), C.c_void_p(stream)),
              "cirrus_full_negative_laplacian_ex")

    def negative_laplacian_same_level(self, tile_level: int, subtree_level: int, launch_tile_types: int, x_channel: int,
                                      Ax_channel: int, calc_diag: bool = False, stream: int = 0) -> None:
        """NegativeLaplacianSameLevel128 (src/GMGSolver.cu:145-201) on the tiles of `tile_level`
        (-1: all tiles) whose subtreeType(subtree_level) is in `launch_tile_types`."""
        check(lib().cirrus_negative_laplacian_same_level(self._h, tile_level, subtree_level, launch_tile_types, x_channel, Ax_channel,
                                                         int(bool(calc_diag)), C.c_void_p(stream)),
              "cirrus_negative_laplacian_same_level")

    def gauss_seidel_sweep(self, level: int, x_channel: int, rhs_channel: int, color: int, stream: int = 0) -> None:
        check(lib().cirrus_gauss_seidel_sweep(self._h, level, x_channel, rhs_channel, color, C.c_void_p(stream)),
              "cirrus_gauss_seidel_sweep")

    def residual_and_restrict(self, level: int, x_channel: int, rhs_channel: int, coarse_channel: int,
                              one_over_alpha: float = 1.0, stream: int = 0) -> None:
        check(lib().cirrus_residual_and_restrict(self._h, level, x_channel, rhs_channel, coarse_channel, one_over_alpha,
                                                 C.c_void_p(stream)), "cirrus_residual_and_restrict")

    def prolongate_and_update(self, fine_level: int, coarse_channel: int, fine_channel: int, prolong_coeff: float = 1.0,
                              stream: int = 0) -> None:
        check(lib().cirrus_prolongate_and_update(self._h, fine_level, coarse_channel, fine_channel, prolong_coeff,
                                                 C.c_void_p(stream)), "cirrus_prolongate_and_update")

    def vcycle(self, x_channel: int, f_channel: int, rhs_channel: int, level_iters: int = 1, coarsest_iters: int = 10,
               stream: int = 0) -> None:
        check(lib().cirrus_vcycle(self._h, x_channel, f_channel, rhs_channel, level_iters, coarsest_iters, C.c_void_p(stream)),
              "cirrus_vcycle")

    def dot(self, a_channel: int, b_channel: int, stream: int = 0) -> float:
        r = C.c_double()
        check(lib().cirrus_dot(self._h, a_channel, b_channel, C.byref(r), C.c_void_p(stream)), "cirrus_dot")
        return r.value

    def clear_neumann_neighbor_faces(self, u_channel: int = U_CHANNEL, stream: int = 0) -> None:
        check(lib().cirrus_clear_neumann_neighbor_faces(self._h, u_channel, C.c_void_p(stream)),
              "cirrus_clear_neumann_neighbor_faces")

    def propagate_to_children(self, channel: int, stream: int = 0) -> None:
        check(lib().cirrus_propagate_to_children(self._h, channel, C.c_void_p(stream)), "cirrus_propagate_to_children")

    def velocity_volume_divergence_on_leafs(self, u_channel: int = U_CHANNEL, div_channel: int = B_CHANNEL,
                                            stream: int = 0) -> None:
        check(lib().cirrus_velocity_volume_divergence_on_leafs(self._h, u_channel, div_channel, C.c_void_p(stream)),
              "cirrus_velocity_volume_divergence_on_leafs")

    def add_gradient_to_face_centers(self, p_channel: int = X_CHANNEL, u_channel: int = U_CHANNEL, stream: int = 0) -> None:
        """AddGradientToFaceCenters: the velocity update from the solved pressure."""
        check(lib().cirrus_add_gradient_to_face_centers(self._h, p_channel, u_channel, C.c_void_p(stream)),
              "cirrus_add_gradient_to_face_centers")

    def projection_rhs(self, stream: int = 0) -> None:
        """b = divergence of the face velocities in channels 6-8, as FluidEuler::project builds it
        after the velocity boundary step (src/FluidEuler.h:583-586, src/FluidEuler.cu:43-60)."""
        self.clear_neumann_neighbor_faces(U_CHANNEL, stream)
        for a in range(3):
            self.propagate_to_children(U_CHANNEL + a, stream)
        self.velocity_volume_divergence_on_leafs(U_CHANNEL, B_CHANNEL, stream)

    def solution_f64(self, stream: int = 0) -> np.ndarray:
        """The last solution in FP64 (the FP64 iterate after a mixed-precision solve)."""
        out = np.empty((self.num_tiles, 512), dtype=np.float64)
        check(lib().cirrus_grid_get_solution_f64(self._h, _ptr(out, C.c_double), C.c_void_p(stream)),
              "cirrus_grid_get_solution_f64")
        return out

    def true_residual(self, b: np.ndarray, stream: int = 0):
        """FP64 ||b - A x|| / ||b|| of the last solution (a float; a list for a batch)."""
        a = np.ascontiguousarray(b, dtype=np.float32).reshape(self.num_tiles * 512)
        r = (C.c_double * self.num_instances)()
        check(lib().cirrus_true_residual(self._h, _ptr(a, C.c_float), r, C.c_void_p(stream)), "cirrus_true_residual")
        return r[0] if self.num_instances == 1 else list(r)


class GMGSolver:
    """Geometric-multigrid-preconditioned CG (the reference's GMGSolver, src/GMGSolver.h:17-52)."""

    def __init__(self, one_over_alpha: float = 1.0, prolong_coeff: float = 1.0, precision: int = PRECISION_FP32,
                 inner_tolerance: float = 1e-7, max_outer_iters: int = 20, warm_start: bool = False):
        self.one_over_alpha = one_over_alpha
        self.prolong_coeff = prolong_coeff
        self.precision = precision
        self.inner_tolerance = inner_tolerance
        self.max_outer_iters = max_outer_iters
        self.warm_start = warm_start
        self.last_result: SolveResult | None = None

    def params(self, max_iters=1000, relative_tolerance=1e-6, level_iters=1, coarsest_iters=10, sync_stride=1,
               is_pure_neumann=False) -> SolveParams:
        p = SolveParams()
        lib().cirrus_solve_params_default(C.byref(p))
        p.max_iters = max_iters
        p.relative_tolerance = relative_tolerance
        p.level_iters = level_iters
        p.coarsest_iters = coarsest_iters
        p.sync_stride = sync_stride
        p.is_pure_neumann = int(bool(is_pure_neumann))
        p.one_over_alpha = self.one_over_alpha
        p.prolong_coeff = self.prolong_coeff
        p.precision = self.precision
        p.warm_start = int(bool(self.warm_start))
        p.inner_tolerance = self.inner_tolerance
        p.max_outer_iters = self.max_outer_iters
        return p

    def solve(self, grid: DeviceGrid, verbose: bool = False, max_iters: int = 1000, relative_tolerance: float = 1e-6,
              level_iters: int = 1, coarsest_iters: int = 10, sync_stride: int = 1, is_pure_neumann: bool = False,
              stream: int = 0) -> tuple[int, float]:
        """Solve -lap(x) = b (b in channel 1, x to channel 0); returns (iters, relative residual).
        As in the reference, channel 1 ends holding the final residual."""
        p = self.params(max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride, is_pure_neumann)
        r = SolveResult()
        check(lib().cirrus_gmg_solve(grid.handle, C.byref(p), C.c_void_p(stream), C.byref(r)), "cirrus_gmg_solve")
        self.last_result = r
        if verbose:
            print(f"GMG-PCG: {r.iters} iters, relative residual {r.rel_residual:.3e}, status {r.status}")
        return r.iters, r.rel_residual

    def solve_batch(self, grid: DeviceGrid, active: Sequence[bool] | None = None, tolerances: Sequence[float] | None = None,
                    pure_neumann: Sequence[bool] | None = None, stream: int = 0, **kw) -> list[tuple[int, float]]:
        """Solve every (active) instance of a batched grid in one graph launch; per-instance
        (iters, relative residual).  Each instance's bits do not depend on the rest of the batch."""
        p = self.params(**kw)
        k = grid.num_instances
        res = (SolveResult * k)()
        act = (C.c_int * k)(*[int(bool(a)) for a in active]) if active is not None else None
        tol = (C.c_double * k)(*tolerances) if tolerances is not None else None
        pn = (C.c_int * k)(*[int(bool(x)) for x in pure_neumann]) if pure_neumann is not None else None
        check(lib().cirrus_gmg_solve_batch(grid.handle, C.byref(p), act, tol, pn, C.c_void_p(stream), res), "cirrus_gmg_solve_batch")
        self.last_results = list(res)
        self.last_result = res[0]
        return [(r.iters, r.rel_residual) for r in res]

    _grids_fn = "cirrus_gmg_solve_grids"

    def solve_grids(self, grids: Sequence[DeviceGrid], stream: int = 0, **kw) -> list[list[tuple[int, float]]]:
        """Solve every instance of several distinct grids at once, each grid's solve on a stream of
        its own (the grids' kernels share the GPU); per grid, per instance (iters, relative
        residual), each bit-identical to that grid's solve_batch."""
        p = self.params(**kw)
        counts = [g.num_instances for g in grids]
        res = (SolveResult * sum(counts))()
        hs = (C.c_void_p * len(grids))(*[g.handle.value for g in grids])
        check(getattr(lib(), self._grids_fn)(hs, len(grids), C.byref(p), C.c_void_p(stream), res), self._grids_fn)
        self.last_results = list(res)
        self.last_result = res[0]
        out, o = [], 0
        for c in counts:
            out.append([(r.iters, r.rel_residual) for r in res[o:o + c]])
            o += c
        return out

    def damped_jacobi_solve(self, grid: DeviceGrid, verbose: bool = False, max_iters: int = 10, relative_tolerance: float = 1e-6,
                            omega: float = 1.0, stream: int = 0) -> tuple[int, float]:
        """GMGSolver::dampedJacobiSolve (src/GMGSolver.cu:449-531): b in channel 1, x to channel 0;
        returns (iterations, relative residual)."""
        it, rel = C.c_int(), C.c_double()
        check(lib().cirrus_damped_jacobi_solve(grid.handle, int(max_iters), float(relative_tolerance), float(omega), C.c_void_p(stream),
                                               C.byref(it), C.byref(rel)), "cirrus_damped_jacobi_solve")
        return it.value, rel.value

    def autotune_sweeps(self, grid: DeviceGrid, stream: int = 0, **kw) -> tuple[int, int]:
        """Time this solver's batched solve of the grid's current right-hand sides for each
        candidate (level_iters, coarsest_iters) and return the fastest pair that converged (pass
        it back as solve_batch(..., level_iters=, coarsest_iters=)).  Sweep counts change the
        iterates -- the reference's bits come only from (1, 10) -- so this is for the
        mixed-precision solver, whose FP64 tolerance fixes the result.  b is restored; x and the
        scratch channels are overwritten."""
        p = self.params(**kw)
        best = SolveParams()
        check(lib().cirrus_grid_autotune_sweeps(grid.handle, C.byref(p), C.c_void_p(stream), C.byref(best)),
              "cirrus_grid_autotune_sweeps")
        return best.level_iters, best.coarsest_iters

    def solve_host(self, grid: DeviceGrid, b: np.ndarray, x_out: np.ndarray, stream: int = 0, **kw) -> tuple[int, float]:
        """End-to-end solve from host buffers (b in, x out; all-tiles order, 512 floats/tile)."""
        p = self.params(**kw)
        r = SolveResult()
        check(lib().cirrus_gmg_solve_host(grid.handle, C.byref(p), _ptr(b, C.c_float), _ptr(x_out, C.c_float),
                                          C.c_void_p(stream), C.byref(r)), "cirrus_gmg_solve_host")
        self.last_result = r
        return r.iters, r.rel_residual

    def solve_host_submit(self, grid: DeviceGrid, b: np.ndarray, x_out: np.ndarray, stream: int = 0, **kw) -> None:
        """Asynchronous end-to-end solve: enqueues the copy of b, the solve and the copy of x into
        x_out on `stream` and returns; solve_host_wait(grid) collects it.  Keep b and x_out
        untouched until then (pinned arrays make the copies asynchronous)."""
        p = self.params(**kw)
        check(lib().cirrus_gmg_solve_host_submit(grid.handle, C.byref(p), _ptr(b, C.c_float), _ptr(x_out, C.c_float),
                                                 C.c_void_p(stream)), "cirrus_gmg_solve_host_submit")
        grid._inflight = (b, x_out)

    def solve_host_wait(self, grid: DeviceGrid) -> list[tuple[int, float]]:
        """Waits for the grid's submitted solve; (iterations, relative residual) per instance."""
        res = (SolveResult * grid.num_instances)()
        check(lib().cirrus_gmg_solve_host_wait(grid.handle, res), "cirrus_gmg_solve_host_wait")
        grid._inflight = None
        return [(r.iters, r.rel_residual) for r in res]


class AMGSolver(GMGSolver):
    """The AMG variant (the reference's AMGSolver, src/AMGSolver.h:20-53): explicit per-cell face
    coefficients with coarse levels formed from the children, its own V-cycle, and GMGSolver's
    PCG around it.  prepare_types_and_coeffs(grid) first (after every change of the cell types);
    solve() then takes b in channel 1 and leaves x in channel 0, using channels 3 and 5 as the
    V-cycle's scratch.  The coefficients live apart from the grid's channels."""

    _grids_fn = "cirrus_amg_solve_grids"

    def prepare_types_and_coeffs(self, grid: DeviceGrid, stream: int = 0) -> None:
        """AMGSolver::prepareTypesAndCoeffs (src/AMGSolver.cu:717-720)."""
        check(lib().cirrus_amg_prepare(grid.handle, float(self.one_over_alpha), C.c_void_p(stream)), "cirrus_amg_prepare")

    def coefficients(self, grid: DeviceGrid, stream: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """((4, n, 512) FP32: x-, y-, z- face off-diagonals and the diagonal; (n, 512) AMG cell types)."""
        n = grid.num_tiles
        co = np.empty((4, n, 512), dtype=np.float32)
        ty = np.empty((n, 512), dtype=np.uint8)
        check(lib().cirrus_amg_coefficients(grid.handle, _ptr(co, C.c_float), _ptr(ty, C.c_uint8), C.c_void_p(stream)),
              "cirrus_amg_coefficients")
        return co, ty

    def vcycle(self, grid: DeviceGrid, x_channel: int = Z_CHANNEL, f_channel: int = R_CHANNEL, tmp_channel: int = AP_CHANNEL,
               rhs_channel: int = TMP_CHANNEL, level_iters: int = 1, coarsest_iters: int = 10, stream: int = 0) -> None:
        """VCycleAMG (src/AMGSolver.cu:610-715)."""
        check(lib().cirrus_amg_vcycle(grid.handle, x_channel, f_channel, tmp_channel, rhs_channel, level_iters, coarsest_iters,
                                      float(self.one_over_alpha), float(self.prolong_coeff), C.c_void_p(stream)), "cirrus_amg_vcycle")

    def solve(self, grid: DeviceGrid, verbose: bool = False, max_iters: int = 1000, relative_tolerance: float = 1e-6,
              level_iters: int = 1, coarsest_iters: int = 10, sync_stride: int = 1, is_pure_neumann: bool = False,
              stream: int = 0) -> tuple[int, float]:
        """AMGSolver::solve (src/AMGSolver.cu:722-853); returns (iters, relative residual)."""
        p = self.params(max_iters, relative_tolerance, level_iters, coarsest_iters, sync_stride, is_pure_neumann)
        r = SolveResult()
        check(lib().cirrus_amg_solve(grid.handle, C.byref(p), C.c_void_p(stream), C.byref(r)), "cirrus_amg_solve")
        self.last_result = r
        if verbose:
            print(f"AMG-PCG: {r.iters} iters, relative residual {r.rel_residual:.3e}, status {r.status}")
        return r.iters, r.rel_residual

    def solve_batch(self, grid: DeviceGrid, active: Sequence[bool] | None = None, tolerances: Sequence[float] | None = None,
                    pure_neumann: Sequence[bool] | None = None, stream: int = 0, **kw) -> list[tuple[int, float]]:
        p = self.params(**kw)
        k = grid.num_instances
        res = (SolveResult * k)()
        act = (C.c_int * k)(*[int(bool(a)) for a in active]) if active is not None else None
        tol = (C.c_double * k)(*tolerances) if tolerances is not None else None
        pn = (C.c_int * k)(*[int(bool(x)) for x in pure_neumann]) if pure_neumann is not None else None
        check(lib().cirrus_amg_solve_batch(grid.handle, C.byref(p), act, tol, pn, C.c_void_p(stream), res), "cirrus_amg_solve_batch")
        self.last_results = list(res)
        self.last_result = res[0]
        return [(r.iters, r.rel_residual) for r in res]

    def solve_host(self, *a, **kw):
        raise NotImplementedError("AMGSolver: solve from device channels (solve / solve_batch)")

    def solve_host_submit(self, *a, **kw):
        raise NotImplementedError("AMGSolver: solve from device channels (solve / solve_batch)")


class Server:
    """Serving loop with continuous batching: sessions (independent problems) of similar size share
    a batched device tile pool; requests that arrive while a pool is busy are merged into its next
    launch (one mixed-precision batched solve, each request warm-started from its session's last
    pressure); `slots` launches run concurrently; pools admitted against an HBM budget (idle pools
    evicted least recently used first).  pool_size 1 keeps every session in a pool of its own."""

    def __init__(self, hbm_budget_bytes: int, slots: int = 4, pool_size: int = 8):
        h = C.c_void_p()
        check(lib().cirrus_server_create_ex(int(hbm_budget_bytes), int(slots), int(pool_size), C.byref(h)), "cirrus_server_create_ex")
        self._h = h
        self._topos = {}
        self._live = {}  # ticket -> (b, x) kept alive until the completion is polled

    def close(self):
        h = getattr(self, "_h", None)
        L = loaded_lib()
        if h is not None and h.value and L is not None:
            L.cirrus_server_destroy(h)
            self._h = None
        self._live.clear()

    def __del__(self):
        self.close()

    def add_session(self, topology: Topology) -> int:
        sid = C.c_int()
        check(lib().cirrus_server_add_session(self._h, topology.handle, C.byref(sid)), "cirrus_server_add_session")
        self._topos[sid.value] = topology
        return sid.value

    def close_session(self, session: int) -> None:
        check(lib().cirrus_server_close_session(self._h, session), "cirrus_server_close_session")
        self._topos.pop(session, None)

    def submit(self, session: int, b: np.ndarray, x_out: np.ndarray, relative_tolerance: float = 1e-6,
               max_iters: int = 1000, inner_tolerance: float = 1e-7) -> int:
        p = SolveParams()
        lib().cirrus_solve_params_default(C.byref(p))
        p.relative_tolerance = relative_tolerance
        p.max_iters = max_iters
        p.inner_tolerance = inner_tolerance
        p.precision = PRECISION_MIXED_FP64
        b = np.ascontiguousarray(b, dtype=np.float32)
        assert x_out.dtype == np.float32 and x_out.flags["C_CONTIGUOUS"]
        t = C.c_uint64()
        check(lib().cirrus_server_submit(self._h, session, C.byref(p), _ptr(b, C.c_float), _ptr(x_out, C.c_float), C.byref(t)),
              "cirrus_server_submit")
        self._live[t.value] = (b, x_out)
        return t.value

    def poll(self, max_items: int = 64, wait_ms: int = 0) -> list[dict]:
        out = (Completion * max_items)()
        n = C.c_int()
        check(lib().cirrus_server_poll(self._h, out, max_items, C.byref(n), wait_ms), "cirrus_server_poll")
        res = []
        for c in out[: n.value]:
            self._live.pop(c.ticket, None)
            res.append({f: getattr(c, f) for f, _ in Completion._fields_})
        return res

    def stats(self) -> dict:
        r, pk, e = C.c_size_t(), C.c_size_t(), C.c_longlong()
        rs, pd = C.c_int(), C.c_int()
        check(lib().cirrus_server_stats(self._h, C.byref(r), C.byref(pk), C.byref(rs), C.byref(pd), C.byref(e)), "cirrus_server_stats")
        nb, nr = C.c_longlong(), C.c_longlong()
        check(lib().cirrus_server_batch_stats(self._h, C.byref(nb), C.byref(nr)), "cirrus_server_batch_stats")
        return {"resident_bytes": r.value, "peak_bytes": pk.value, "resident_sessions": rs.value, "pending": pd.value,
                "evictions": e.value, "launches": nb.value, "requests": nr.value}


class Holder:
    """A tile-holder file in memory: the reference's checkpoint / interchange format of a grid's
    tiles (IOFunc::WriteHAHostTileHolderToFile / ReadHAHostTileHolderFromFile,
    src/PoissonIOFunc.cu:38-121).  Tiles are listed level by level in file order."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    @classmethod
    def read(cls, path: str) -> "Holder":
        h = C.c_void_p()
        check(lib().cirrus_holder_read(str(path).encode(), C.byref(h)), "cirrus_holder_read")
        return cls(h)

    @classmethod
    def from_grid(cls, topology: Topology, grid: DeviceGrid, tile_types: int = LEAF | NONLEAF | GHOST) -> "Holder":
        """getHostTileHolder(tile_types): the grid's tiles of those types with channels 0..8 and
        cell types (synchronous)."""
        h = C.c_void_p()
        check(lib().cirrus_holder_from_grid(topology.handle, grid.handle, int(tile_types), C.byref(h)), "cirrus_holder_from_grid")
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        L = loaded_lib()
        if h is not None and h.value and L is not None:
            L.cirrus_holder_destroy(h)
            self._h = None

    def write(self, path: str) -> None:
        check(lib().cirrus_holder_write(self._h, str(path).encode()), "cirrus_holder_write")

    def info(self) -> dict:
        h0, nl, ml, nt = C.c_double(), C.c_int(), C.c_int(), C.c_int()
        check(lib().cirrus_holder_info(self._h, C.byref(h0), C.byref(nl), C.byref(ml), C.byref(nt)), "cirrus_holder_info")
        return {"h0": h0.value, "num_layers": nl.value, "max_level": ml.value, "num_tiles": nt.value}

    @property
    def num_tiles(self) -> int:
        return self.info()["num_tiles"]

    def tiles(self) -> np.ndarray:
        out = np.empty((self.num_tiles, 5), dtype=np.int32)
        check(lib().cirrus_holder_tiles(self._h, _ptr(out, C.c_int32)), "cirrus_holder_tiles")
        return out

    def cell_types(self) -> np.ndarray:
        out = np.empty((self.num_tiles, 512), dtype=np.uint8)
        check(lib().cirrus_holder_cell_types(self._h, _ptr(out, C.c_uint8)), "cirrus_holder_cell_types")
        return out

    def channel(self, c: int) -> np.ndarray:
        out = np.empty((self.num_tiles, 512), dtype=np.float32)
        check(lib().cirrus_holder_channel(self._h, int(c), _ptr(out, C.c_float)), "cirrus_holder_channel")
        return out

    def to_topology(self, levels_log2_hash: Sequence[int] = FLUID_EULER_LOG2_HASH) -> tuple[Topology, np.ndarray]:
        """setTilesFromHolder + compressHost into a new Topology; also returns each holder tile's
        index in the topology's all-tiles order."""
        nl = len(levels_log2_hash)
        arr = (C.c_uint32 * nl)(*levels_log2_hash)
        order = np.empty(self.num_tiles, dtype=np.int32)
        h = C.c_void_p()
        check(lib().cirrus_topology_from_holder(self._h, arr, nl, C.byref(h), _ptr(order, C.c_int32)), "cirrus_topology_from_holder")
        t = Topology.__new__(Topology)
        t.num_layers = nl
        t.h0 = self.info()["h0"]
        t._h = h
        return t, order

    def load_into(self, grid: DeviceGrid, order: np.ndarray, channels: Sequence[int] = (0,), stream: int = 0) -> None:
        """Copy the holder's channels into the grid's tiles at `order` (from to_topology)."""
        mask = 0
        for c in channels:
            mask |= 1 << int(c)
        o = np.ascontiguousarray(order, dtype=np.int32)
        check(lib().cirrus_grid_load_holder(grid.handle, self._h, _ptr(o, C.c_int32), mask, C.c_void_p(stream)), "cirrus_grid_load_holder")


class DeviceTopology:
    """The octree construction on the GPU (RefineLeafsOneStep, CoarsenStep, SpawnGhostTiles,
    compressHost/syncHostAndDevice, CalcCellTypesFromLeafs): tables, statuses and cell types in
    device memory, bit-exact with Topology and the reference."""

    def __init__(self, h0: float = 1.0 / 8, levels_log2_hash: Sequence[int] = FLUID_EULER_LOG2_HASH):
        self.num_layers = len(levels_log2_hash)
        self.h0 = float(h0)
        self.log2_hash = tuple(levels_log2_hash)
        arr = (C.c_uint32 * self.num_layers)(*levels_log2_hash)
        h = C.c_void_p()
        check(lib().cirrus_dtopology_create(self.num_layers, arr, self.h0, C.byref(h)), "cirrus_dtopology_create")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        L = loaded_lib()
        if h is not None and h.value and L is not None:
            L.cirrus_dtopology_destroy(h)
            self._h = None

    def set_tiles(self, level: int, coords: np.ndarray, types) -> None:
        xyz = np.ascontiguousarray(coords, dtype=np.int32).reshape(-1, 3)
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(types, dtype=np.uint8), (xyz.shape[0],)))
        check(lib().cirrus_dtopology_set_tiles(self._h, level, _ptr(xyz, C.c_int32), _ptr(t, C.c_uint8), xyz.shape[0]),
              "cirrus_dtopology_set_tiles")

    def compress(self) -> None:
        check(lib().cirrus_dtopology_compress(self._h), "cirrus_dtopology_compress")

    def spawn_ghost_tiles(self) -> None:
        check(lib().cirrus_dtopology_spawn_ghost_tiles(self._h), "cirrus_dtopology_spawn_ghost_tiles")

    def refine_leafs_one_step(self, masks) -> list[int]:
        keep, ptrs, dims = _mask_args(masks, self.num_layers)
        out = (C.c_int * self.num_layers)()
        check(lib().cirrus_dtopology_refine_leafs_one_step(self._h, ptrs, dims, out), "cirrus_dtopology_refine_leafs_one_step")
        del keep
        return list(out)

    def iterative_refine(self, masks) -> None:
        keep, ptrs, dims = _mask_args(masks, self.num_layers)
        check(lib().cirrus_dtopology_iterative_refine(self._h, ptrs, dims), "cirrus_dtopology_iterative_refine")
        del keep

    def coarsen_step(self, masks) -> list[int]:
        """CoarsenStep: a LEAF tile whose mask entry is set has target level - 1."""
        keep, ptrs, dims = _mask_args(masks, self.num_layers)
        out = (C.c_int * self.num_layers)()
        check(lib().cirrus_dtopology_coarsen_step(self._h, ptrs, dims, out), "cirrus_dtopology_coarsen_step")
        del keep
        return list(out)

    def set_cell_types(self, ctypes: np.ndarray) -> None:
        a = np.ascontiguousarray(ctypes, dtype=np.uint8).reshape(self.num_tiles, 512)
        check(lib().cirrus_dtopology_set_cell_types(self._h, _ptr(a, C.c_uint8)), "cirrus_dtopology_set_cell_types")

    def calc_cell_types_from_leafs(self) -> None:
        check(lib().cirrus_dtopology_calc_cell_types_from_leafs(self._h), "cirrus_dtopology_calc_cell_types_from_leafs")

    @property
    def num_tiles(self) -> int:
        n = C.c_int()
        check(lib().cirrus_dtopology_num_tiles(self._h, C.byref(n)), "cirrus_dtopology_num_tiles")
        return n.value

    @property
    def max_level(self) -> int:
        n = C.c_int()
        check(lib().cirrus_dtopology_max_level(self._h, C.byref(n)), "cirrus_dtopology_max_level")
        return n.value

    def tiles(self) -> np.ndarray:
        out = np.empty((self.num_tiles, 5), dtype=np.int32)
        check(lib().cirrus_dtopology_tiles(self._h, _ptr(out, C.c_int32)), "cirrus_dtopology_tiles")
        return out

    def hash_slots(self) -> np.ndarray:
        out = np.empty(self.num_tiles, dtype=np.int32)
        check(lib().cirrus_dtopology_hash_slots(self._h, _ptr(out, C.c_int32)), "cirrus_dtopology_hash_slots")
        return out

    def cell_types(self) -> np.ndarray:
        out = np.empty((self.num_tiles, 512), dtype=np.uint8)
        check(lib().cirrus_dtopology_cell_types(self._h, _ptr(out, C.c_uint8)), "cirrus_dtopology_cell_types")
        return out

    def statuses(self) -> np.ndarray:
        out = np.empty(self.num_tiles, dtype=np.int32)
        check(lib().cirrus_dtopology_statuses(self._h, _ptr(out, C.c_int32)), "cirrus_dtopology_statuses")
        return out

    def to_topology(self) -> Topology:
        h = C.c_void_p()
        check(lib().cirrus_dtopology_to_topology(self._h, C.byref(h)), "cirrus_dtopology_to_topology")
        t = Topology.__new__(Topology)
        t.num_layers = self.num_layers
        t.h0 = self.h0
        t._h = h
        return t
