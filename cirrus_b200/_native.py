"""ctypes binding of libcirrus_b200.so (the C ABI of include/cirrus_b200.h).

The library is loaded from cirrus_b200/_lib/; if it is missing it is built with nvcc (see
cirrus_b200/build.py).  There is no fallback implementation: a failure to load or a missing
CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

_LIB = None
_LOCK = threading.Lock()


class CirrusError(RuntimeError):
    """A C-ABI call returned a status other than CIRRUS_OK."""

    def __init__(self, status: int, func: str):
        self.status = status
        msg = lib().cirrus_status_string(status).decode() if _LIB is not None else str(status)
        super().__init__(f"{func}: {msg} (status {status})")


CIRRUS_OK = 0
CIRRUS_ERR_NOT_CONVERGED = 5
CIRRUS_ERR_NO_DEVICE = 8

c_int_p = C.POINTER(C.c_int)
c_i32_p = C.POINTER(C.c_int32)
c_u8_p = C.POINTER(C.c_uint8)
c_f32_p = C.POINTER(C.c_float)
c_f64_p = C.POINTER(C.c_double)
LEVEL_TARGET_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int)


class GridDesc(C.Structure):
    _fields_ = [
        ("h0", C.c_double),
        ("num_layers", C.c_int),
        ("log2_hash", C.POINTER(C.c_uint32)),
        ("tiles_per_level", C.POINTER(C.c_int32)),
        ("coords", C.POINTER(C.c_int32)),
        ("types", C.POINTER(C.c_uint8)),
        ("cell_types", C.POINTER(C.c_uint8)),
        ("b", C.POINTER(C.c_float)),
        ("x0", C.POINTER(C.c_float)),
    ]


class SolveParams(C.Structure):
    _fields_ = [
        ("max_iters", C.c_int),
        ("relative_tolerance", C.c_double),
        ("level_iters", C.c_int),
        ("coarsest_iters", C.c_int),
        ("sync_stride", C.c_int),
        ("is_pure_neumann", C.c_int),
        ("one_over_alpha", C.c_float),
        ("prolong_coeff", C.c_float),
        ("precision", C.c_int),
        ("warm_start", C.c_int),
        ("inner_tolerance", C.c_double),
        ("max_outer_iters", C.c_int),
    ]


class SolveResult(C.Structure):
    _fields_ = [
        ("iters", C.c_int),
        ("outer_iters", C.c_int),
        ("rel_residual", C.c_double),
        ("true_rel_residual", C.c_double),
        ("status", C.c_int),
        ("kernel_launches", C.c_longlong),
    ]


class Completion(C.Structure):
    _fields_ = [
        ("ticket", C.c_uint64),
        ("session", C.c_int),
        ("slot", C.c_int),
        ("status", C.c_int),
        ("iters", C.c_int),
        ("outer_iters", C.c_int),
        ("warm", C.c_int),
        ("rel_residual", C.c_double),
        ("latency_ms", C.c_double),
        ("device_ms", C.c_double),
        ("batch", C.c_int),
    ]


# name -> (restype, argtypes); status-returning functions use c_int
_PROTOS = {
    "cirrus_status_string": (C.c_char_p, [C.c_int]),
    "cirrus_version": (C.c_char_p, []),
    "cirrus_topology_create": (C.c_int, [C.c_int, C.POINTER(C.c_uint32), C.c_double, C.POINTER(C.c_void_p)]),
    "cirrus_topology_destroy": (None, [C.c_void_p]),
    "cirrus_topology_set_tile": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "cirrus_topology_compress": (C.c_int, [C.c_void_p]),
    "cirrus_topology_spawn_ghost_tiles": (C.c_int, [C.c_void_p]),
    "cirrus_topology_refine_leafs_one_step": (C.c_int, [C.c_void_p, LEVEL_TARGET_FN, C.c_void_p, c_int_p]),
    "cirrus_topology_iterative_refine": (C.c_int, [C.c_void_p, LEVEL_TARGET_FN, C.c_void_p]),
    "cirrus_topology_iterative_refine_masks": (C.c_int, [C.c_void_p, C.POINTER(c_u8_p), c_int_p]),
    "cirrus_topology_num_tiles": (C.c_int, [C.c_void_p, c_int_p]),
    "cirrus_topology_max_level": (C.c_int, [C.c_void_p, c_int_p]),
    "cirrus_topology_tiles": (C.c_int, [C.c_void_p, c_i32_p]),
    "cirrus_topology_hash_slots": (C.c_int, [C.c_void_p, c_i32_p]),
    "cirrus_topology_set_cell_types": (C.c_int, [C.c_void_p, c_u8_p]),
    "cirrus_topology_cell_types": (C.c_int, [C.c_void_p, c_u8_p]),
    "cirrus_topology_calc_cell_types_from_leafs": (C.c_int, [C.c_void_p]),
    "cirrus_topology_neighbor_tiles": (C.c_int, [C.c_void_p, c_i32_p]),
    "cirrus_grid_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "cirrus_grid_create_batch": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    "cirrus_grid_num_instances": (C.c_int, [C.c_void_p, c_int_p]),
    "cirrus_grid_instance_info": (C.c_int, [C.c_void_p, C.c_int, c_int_p, C.POINTER(C.c_int64)]),
    "cirrus_grid_set_channel_instance": (C.c_int, [C.c_void_p, C.c_int, C.c_int, c_f32_p, C.c_void_p]),
    "cirrus_grid_get_channel_instance": (C.c_int, [C.c_void_p, C.c_int, C.c_int, c_f32_p, C.c_void_p]),
    "cirrus_grid_destroy": (None, [C.c_void_p]),
    "cirrus_grid_num_tiles": (C.c_int, [C.c_void_p, c_int_p]),
    "cirrus_grid_device_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "cirrus_grid_dof": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "cirrus_grid_set_channel": (C.c_int, [C.c_void_p, C.c_int, c_f32_p, C.c_void_p]),
    "cirrus_grid_get_channel": (C.c_int, [C.c_void_p, C.c_int, c_f32_p, C.c_void_p]),
    "cirrus_grid_channel_ptr": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "cirrus_grid_copy_channel": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_topology_import_tiles": (C.c_int, [C.c_void_p, c_i32_p, C.c_int]),
    "cirrus_grid_set_tile_pointers": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "cirrus_grid_gather_tiles": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, C.c_void_p]),
    "cirrus_grid_scatter_tiles": (C.c_int, [C.c_void_p, C.c_int, C.c_size_t, C.c_void_p]),
    "cirrus_grid_compare_tile_cell_types": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.POINTER(C.c_int),
                                                       C.POINTER(C.c_uint8)]),
    "cirrus_gather_tile_bytes": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_size_t, C.POINTER(C.c_uint8), C.c_void_p]),
    "cirrus_holder_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "cirrus_holder_write": (C.c_int, [C.c_void_p, C.c_char_p]),
    "cirrus_holder_destroy": (None, [C.c_void_p]),
    "cirrus_holder_info": (C.c_int, [C.c_void_p, c_f64_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cirrus_holder_tiles": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "cirrus_holder_cell_types": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "cirrus_holder_channel": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    "cirrus_topology_from_holder": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.c_int, C.POINTER(C.c_void_p),
                                              C.POINTER(C.c_int32)]),
    "cirrus_holder_from_grid": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "cirrus_grid_load_holder": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_uint32, C.c_void_p]),
    "cirrus_dtopology_create": (C.c_int, [C.c_int, C.POINTER(C.c_uint32), C.c_double, C.POINTER(C.c_void_p)]),
    "cirrus_dtopology_destroy": (None, [C.c_void_p]),
    "cirrus_dtopology_set_tiles": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_uint8), C.c_int]),
    "cirrus_dtopology_compress": (C.c_int, [C.c_void_p]),
    "cirrus_dtopology_spawn_ghost_tiles": (C.c_int, [C.c_void_p]),
    "cirrus_dtopology_refine_leafs_one_step": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_int),
                                                         C.POINTER(C.c_int)]),
    "cirrus_dtopology_iterative_refine": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_int)]),
    "cirrus_dtopology_coarsen_step": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cirrus_dtopology_set_cell_types": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "cirrus_dtopology_calc_cell_types_from_leafs": (C.c_int, [C.c_void_p]),
    "cirrus_dtopology_num_tiles": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "cirrus_dtopology_max_level": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "cirrus_dtopology_tiles": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "cirrus_dtopology_hash_slots": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "cirrus_dtopology_cell_types": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "cirrus_dtopology_statuses": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "cirrus_dtopology_to_topology": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "cirrus_server_create_ex": (C.c_int, [C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "cirrus_server_batch_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "cirrus_grid_set_launch_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "cirrus_grid_get_launch_mode": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "cirrus_full_negative_laplacian": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_full_negative_laplacian_ex": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_negative_laplacian_same_level": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                                       C.c_void_p]),
    "cirrus_gauss_seidel_sweep": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_residual_and_restrict": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "cirrus_prolongate_and_update": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "cirrus_vcycle": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_dot": (C.c_int, [C.c_void_p, C.c_int, C.c_int, c_f64_p, C.c_void_p]),
    "cirrus_leaf_dot_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, c_f64_p, C.c_void_p]),
    "cirrus_clear_neumann_neighbor_faces": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "cirrus_propagate_to_children": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "cirrus_velocity_volume_divergence_on_leafs": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_add_gradient_to_face_centers": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_solve_params_default": (None, [C.POINTER(SolveParams)]),
    "cirrus_gmg_solve": (C.c_int, [C.c_void_p, C.POINTER(SolveParams), C.c_void_p, C.POINTER(SolveResult)]),
    "cirrus_gmg_solve_batch": (C.c_int, [C.c_void_p, C.POINTER(SolveParams), c_int_p, c_f64_p, c_int_p, C.c_void_p,
                                         C.POINTER(SolveResult)]),
    "cirrus_gmg_solve_host": (C.c_int, [C.c_void_p, C.POINTER(SolveParams), c_f32_p, c_f32_p, C.c_void_p, C.POINTER(SolveResult)]),
    "cirrus_amg_prepare": (C.c_int, [C.c_void_p, C.c_float, C.c_void_p]),
    "cirrus_amg_coefficients": (C.c_int, [C.c_void_p, c_f32_p, C.POINTER(C.c_uint8), C.c_void_p]),
    "cirrus_amg_vcycle": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                    C.c_void_p]),
    "cirrus_amg_solve": (C.c_int, [C.c_void_p, C.POINTER(SolveParams), C.c_void_p, C.POINTER(SolveResult)]),
    "cirrus_amg_solve_batch": (C.c_int, [C.c_void_p, C.POINTER(SolveParams), c_int_p, c_f64_p, c_int_p, C.c_void_p,
                                         C.POINTER(SolveResult)]),
    "cirrus_gmg_solve_host_submit": (C.c_int, [C.c_void_p, C.POINTER(SolveParams), c_f32_p, c_f32_p, C.c_void_p]),
    "cirrus_gmg_solve_host_wait": (C.c_int, [C.c_void_p, C.POINTER(SolveResult)]),
    "cirrus_server_create": (C.c_int, [C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]),
    "cirrus_server_destroy": (None, [C.c_void_p]),
    "cirrus_server_add_session": (C.c_int, [C.c_void_p, C.c_void_p, c_int_p]),
    "cirrus_server_close_session": (C.c_int, [C.c_void_p, C.c_int]),
    "cirrus_server_submit": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(SolveParams), c_f32_p, c_f32_p, C.POINTER(C.c_uint64)]),
    "cirrus_server_poll": (C.c_int, [C.c_void_p, C.POINTER(Completion), C.c_int, c_int_p, C.c_int]),
    "cirrus_server_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), c_int_p, c_int_p,
                                      C.POINTER(C.c_longlong)]),
    "cirrus_grid_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "cirrus_damped_jacobi_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_float, C.c_void_p, C.POINTER(C.c_int),
                                             C.POINTER(C.c_double)]),
    "cirrus_grid_create_from_desc": (C.c_int, [C.POINTER(GridDesc), C.POINTER(C.c_void_p)]),
    "cirrus_grid_autotune_sweeps": (C.c_int, [C.c_void_p, C.POINTER(SolveParams), C.c_void_p, C.POINTER(SolveParams)]),
    "cirrus_gmg_solve_grids": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(SolveParams), C.c_void_p, C.POINTER(SolveResult)]),
    "cirrus_amg_solve_grids": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(SolveParams), C.c_void_p, C.POINTER(SolveResult)]),
    "cirrus_grid_set_launch_shape": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "cirrus_grid_get_launch_shape": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "cirrus_bench_launch": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "cirrus_true_residual": (C.c_int, [C.c_void_p, c_f32_p, c_f64_p, C.c_void_p]),
    "cirrus_grid_get_solution_f64": (C.c_int, [C.c_void_p, c_f64_p, C.c_void_p]),
}


def library_path() -> Path:
    from . import build as _build

    return _build.LIB


def lib():
    """Load (building first if needed) and return the native library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        from . import build as _build

        path = _build.LIB
        if not path.exists():
            _build.build()
        handle = C.CDLL(str(path))
        for name, (res, args) in _PROTOS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
        return _LIB


def loaded_lib():
    """The native library if it is loaded, else None (for finalizers: during interpreter shutdown
    module globals may already be cleared, and nothing should be loaded then)."""
    return _LIB


def check(status: int, func: str) -> None:
    if status != CIRRUS_OK:
        raise CirrusError(status, func)


def exported_symbols() -> list[str]:
    return sorted(_PROTOS)
