"""Python access to the two checkers of the Poisson path.  TEST INFRASTRUCTURE ONLY.

* `CpuOracle`: oracle/cirrus_oracle.cpp, the CPU restatement of the reference algorithm
  (FP32 mirror of the reference arithmetic, and FP64).
* `RefHarness`: oracle/_ref/libcirrus_ref.so, the reference's own CUDA sources compiled by
  oracle/build_ref.sh around oracle/ref_harness.cu (needs a GPU to run).  It links nothing of
  the product.
* `RefHarness.solve_dropin` / `damped_jacobi_dropin`: oracle/_ref/libcirrus_ref_dropin.so, the
  product's drop-in header run on a reference grid (loads the product library; tests only).

Only tests/, __graft_entry__.smoke() and bench.py's reference/CPU-baseline legs import this
module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "libcirrus_oracle.so"
REF_LIB = HERE / "_ref" / "libcirrus_ref.so"
REF_DROPIN_LIB = HERE / "_ref" / "libcirrus_ref_dropin.so"

P = C.c_void_p
i32p = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def build_oracle(force: bool = False) -> Path:
    src = HERE / "cirrus_oracle.cpp"
    if force or not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["bash", str(HERE / "build_oracle.sh")], check=True, capture_output=True)
    return ORACLE_LIB


def build_ref(force: bool = False, reference_dir: str | None = None) -> Path | None:
    """Compile the reference harness when the reference tree is present; returns None otherwise."""
    # the reference tree: an explicit argument, CIRRUS_REFERENCE_DIR, else `reference` beside
    # this repository
    ref = Path(reference_dir or os.environ.get("CIRRUS_REFERENCE_DIR", str(HERE.parent.parent / "reference")))
    if not (ref / "src").is_dir():
        return REF_LIB if REF_LIB.exists() else None
    deps = [HERE / "ref_harness.cu", HERE / "ref_dropin_harness.cu", HERE / "build_ref.sh",
            *sorted((HERE.parent / "include").glob("*.h*"))]
    outs = [REF_LIB, REF_DROPIN_LIB]
    if force or not all(o.exists() for o in outs) or any(o.stat().st_mtime < d.stat().st_mtime for o in outs for d in deps):
        env = dict(os.environ, CIRRUS_REFERENCE_DIR=str(ref))
        subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True, capture_output=True, env=env)
    return REF_LIB


def _mask_args(masks, num_layers):
    keep = []
    ptrs = (u8p * num_layers)()
    dims = (C.c_int * (3 * num_layers))()
    for l in range(num_layers):
        m = masks[l] if l < len(masks) else None
        if m is None:
            ptrs[l] = u8p()
            continue
        a = np.ascontiguousarray(m, dtype=np.uint8)
        keep.append(a)
        ptrs[l] = _p(a, C.c_uint8)
        dims[3 * l], dims[3 * l + 1], dims[3 * l + 2] = a.shape
    return keep, ptrs, dims


# ================================================================================ CPU oracle
_OLIB = None


def oracle_lib():
    global _OLIB
    if _OLIB is None:
        build_oracle()
        L = C.CDLL(str(ORACLE_LIB))
        protos = {
            "ocx_topo_create": (P, [C.c_int, C.POINTER(C.c_uint32)]),
            "ocx_topo_destroy": (None, [P]),
            "ocx_topo_set_tile": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ocx_topo_compress_sync": (None, [P]),
            "ocx_topo_spawn_ghosts": (None, [P]),
            "ocx_topo_refine_step": (C.c_int, [P, C.POINTER(u8p), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "ocx_topo_iterative_refine": (None, [P, C.POINTER(u8p), C.POINTER(C.c_int)]),
            "ocx_topo_num_tiles": (C.c_int, [P]),
            "ocx_topo_tiles": (None, [P, i32p]),
            "ocx_topo_slots": (None, [P, i32p]),
            "ocx_flat_create": (P, [i32p, C.c_int, C.c_int]),
            "ocx_flat_destroy": (None, [P]),
            "ocx_flat_set_ctypes": (None, [P, u8p]),
            "ocx_flat_get_ctypes": (None, [P, u8p]),
            "ocx_flat_calc_cell_types": (None, [P]),
            "ocx_flat_neighbors": (None, [P, i32p]),
            "ocx_flat_rhs": (None, [P, f32p, f32p, f32p, f32p]),
            "ocx_flat_gradient": (None, [P, f32p, f32p, f32p, f32p]),
            "ocx_set_channel": (None, [P, C.c_int, C.c_int, f64p]),
            "ocx_get_channel": (None, [P, C.c_int, C.c_int, f64p]),
            "ocx_set_channel_f32": (None, [P, C.c_int, f32p]),
            "ocx_get_channel_f32": (None, [P, C.c_int, f32p]),
            "ocx_full_lap": (None, [P, C.c_int, C.c_int, C.c_int]),
            "ocx_full_lap_diag": (None, [P, C.c_int, C.c_int, C.c_int]),
            "ocx_lap_same_level": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ocx_gs_sweep": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ocx_residual_restrict": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ocx_prolongate": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ocx_vcycle": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ocx_dot": (C.c_double, [P, C.c_int, C.c_int, C.c_int]),
            "ocx_solve": (C.c_int, [P, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, f64p, f64p,
                                    C.c_int, C.POINTER(C.c_int)]),
            "ocx_damped_jacobi": (C.c_int, [P, C.c_int, C.c_int, C.c_double, C.c_double, f64p]),
            "ocx_amg_prepare": (None, [P, C.c_int, C.c_double]),
            "ocx_amg_coeffs": (None, [P, C.c_int, C.c_int, f64p]),
            "ocx_amg_types": (None, [P, C.c_int, u8p]),
            "ocx_amg_vcycle": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]),
            "ocx_amg_solve": (C.c_int, [P, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                        f64p]),
            "ocx_num_threads": (C.c_int, []),
            "ocx_set_threads": (None, [C.c_int]),
        }
        for k, (r, a) in protos.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _OLIB = L
    return _OLIB


class OracleTopology:
    """The reference's topology construction restated (hash tables, refine, ghosts)."""

    def __init__(self, log2_hash):
        self.num_layers = len(log2_hash)
        arr = (C.c_uint32 * self.num_layers)(*log2_hash)
        self.h = oracle_lib().ocx_topo_create(self.num_layers, arr)

    def __del__(self):
        if getattr(self, "h", None):
            oracle_lib().ocx_topo_destroy(self.h)
            self.h = None

    def set_tile(self, level, c, t):
        assert oracle_lib().ocx_topo_set_tile(self.h, level, int(c[0]), int(c[1]), int(c[2]), t) == 0

    def compress_sync(self):
        oracle_lib().ocx_topo_compress_sync(self.h)

    def spawn_ghosts(self):
        oracle_lib().ocx_topo_spawn_ghosts(self.h)

    def iterative_refine(self, masks):
        keep, ptrs, dims = _mask_args(masks, self.num_layers)
        oracle_lib().ocx_topo_iterative_refine(self.h, ptrs, dims)
        del keep

    def tiles(self):
        n = oracle_lib().ocx_topo_num_tiles(self.h)
        out = np.empty((n, 5), dtype=np.int32)
        oracle_lib().ocx_topo_tiles(self.h, _p(out, C.c_int32))
        return out

    def slots(self):
        n = oracle_lib().ocx_topo_num_tiles(self.h)
        out = np.empty(n, dtype=np.int32)
        oracle_lib().ocx_topo_slots(self.h, _p(out, C.c_int32))
        return out


def oracle_topology(w):
    """Build a workload's topology with the oracle's restatement."""
    t = OracleTopology(w.log2_hash)
    for r in w.roots:
        t.set_tile(0, r, 1)
    t.compress_sync()
    t.spawn_ghosts()
    t.iterative_refine(w.masks)
    return t


class CpuOracle:
    """Flat solver view: tiles (n,5) in all-tiles order plus cell types."""

    FP32, FP64 = 0, 1

    def __init__(self, tiles: np.ndarray, num_layers: int = 10):
        t = np.ascontiguousarray(tiles, dtype=np.int32)
        self.n = t.shape[0]
        self.h = oracle_lib().ocx_flat_create(_p(t, C.c_int32), self.n, num_layers)

    def __del__(self):
        if getattr(self, "h", None):
            oracle_lib().ocx_flat_destroy(self.h)
            self.h = None

    def set_ctypes(self, ct):
        a = np.ascontiguousarray(ct, dtype=np.uint8).reshape(self.n * 512)
        oracle_lib().ocx_flat_set_ctypes(self.h, _p(a, C.c_uint8))

    def ctypes(self):
        out = np.empty((self.n, 512), dtype=np.uint8)
        oracle_lib().ocx_flat_get_ctypes(self.h, _p(out, C.c_uint8))
        return out

    def calc_cell_types(self):
        oracle_lib().ocx_flat_calc_cell_types(self.h)

    def neighbors(self):
        out = np.empty((self.n, 6), dtype=np.int32)
        oracle_lib().ocx_flat_neighbors(self.h, _p(out, C.c_int32))
        return out

    def rhs(self, velocity: np.ndarray) -> np.ndarray:
        u = [np.ascontiguousarray(velocity[a], dtype=np.float32).copy() for a in range(3)]
        b = np.zeros((self.n, 512), dtype=np.float32)
        oracle_lib().ocx_flat_rhs(self.h, _p(u[0], C.c_float), _p(u[1], C.c_float), _p(u[2], C.c_float), _p(b, C.c_float))
        return b

    def add_gradient(self, p: np.ndarray, velocity: np.ndarray):
        """AddGradientToFaceCenters on copies: returns (p with GHOST cells propagated, u, v, w)."""
        pp = np.ascontiguousarray(p, dtype=np.float32).copy()
        u = [np.ascontiguousarray(velocity[a], dtype=np.float32).copy() for a in range(3)]
        oracle_lib().ocx_flat_gradient(self.h, _p(pp, C.c_float), _p(u[0], C.c_float), _p(u[1], C.c_float), _p(u[2], C.c_float))
        return pp, u

    def set_channel(self, prec, c, data):
        a = np.ascontiguousarray(data, dtype=np.float64).reshape(self.n * 512)
        oracle_lib().ocx_set_channel(self.h, prec, c, _p(a, C.c_double))

    def get_channel(self, prec, c):
        out = np.empty((self.n, 512), dtype=np.float64)
        oracle_lib().ocx_get_channel(self.h, prec, c, _p(out, C.c_double))
        return out

    def set_channel_f32(self, c, data):
        a = np.ascontiguousarray(data, dtype=np.float32).reshape(self.n * 512)
        oracle_lib().ocx_set_channel_f32(self.h, c, _p(a, C.c_float))

    def get_channel_f32(self, c):
        out = np.empty((self.n, 512), dtype=np.float32)
        oracle_lib().ocx_get_channel_f32(self.h, c, _p(out, C.c_float))
        return out

    def full_lap(self, prec, xc, yc):
        oracle_lib().ocx_full_lap(self.h, prec, xc, yc)

    def full_lap_diag(self, prec, xc, yc):
        oracle_lib().ocx_full_lap_diag(self.h, prec, xc, yc)

    def lap_same_level(self, prec, tile_level, subtree_level, types, xc, yc, diag=False):
        oracle_lib().ocx_lap_same_level(self.h, prec, tile_level, subtree_level, types, xc, yc, int(diag))

    def gs_sweep(self, prec, level, xc, rc, color):
        oracle_lib().ocx_gs_sweep(self.h, prec, level, xc, rc, color)

    def residual_restrict(self, prec, level, xc, rhsc, coarsec):
        oracle_lib().ocx_residual_restrict(self.h, prec, level, xc, rhsc, coarsec)

    def prolongate(self, prec, level, cxc, fxc):
        oracle_lib().ocx_prolongate(self.h, prec, level, cxc, fxc)

    def vcycle(self, prec, xc=4, fc=1, rhsc=3, level_iters=1, coarsest_iters=10):
        oracle_lib().ocx_vcycle(self.h, prec, xc, fc, rhsc, level_iters, coarsest_iters)

    def dot(self, prec, a, b):
        return oracle_lib().ocx_dot(self.h, prec, a, b)

    def solve(self, prec, max_iters=1000, tol=1e-6, level_iters=1, coarsest_iters=10, sync_stride=1, pure_neumann=False):
        rel = C.c_double()
        hist = np.zeros(max(max_iters, 1), dtype=np.float64)
        hl = C.c_int()
        it = oracle_lib().ocx_solve(self.h, prec, max_iters, tol, level_iters, coarsest_iters, sync_stride,
                                    int(pure_neumann), C.byref(rel), _p(hist, C.c_double), hist.size, C.byref(hl))
        return it, rel.value, hist[:hl.value].copy()

    def damped_jacobi(self, prec, max_iters=10, tol=1e-6, omega=1.0):
        """GMGSolver::dampedJacobiSolve restated: b in channel 1; returns (iterations, relative residual)."""
        rel = C.c_double()
        it = oracle_lib().ocx_damped_jacobi(self.h, prec, max_iters, tol, omega, C.byref(rel))
        return it, rel.value


    # AMG variant (src/AMGSolver.cu), parity unpinned: the reference's AMG file does not build here
    def amg_prepare(self, prec, one_over_alpha=1.0):
        oracle_lib().ocx_amg_prepare(self.h, prec, one_over_alpha)

    def amg_coefficients(self, prec):
        """(4, n, 512): off-diagonal coefficients of the x-, y-, z- faces and the diagonal."""
        out = np.empty((4, self.n, 512), dtype=np.float64)
        for k in range(4):
            oracle_lib().ocx_amg_coeffs(self.h, prec, k, _p(out[k], C.c_double))
        return out

    def amg_types(self, prec):
        out = np.empty((self.n, 512), dtype=np.uint8)
        oracle_lib().ocx_amg_types(self.h, prec, _p(out, C.c_uint8))
        return out

    def amg_vcycle(self, prec, xc=4, fc=1, tmpc=3, rhsc=5, level_iters=1, coarsest_iters=10, one_over_alpha=1.0, prolong_coeff=1.0):
        oracle_lib().ocx_amg_vcycle(self.h, prec, xc, fc, tmpc, rhsc, level_iters, coarsest_iters, one_over_alpha, prolong_coeff)

    def amg_solve(self, prec, max_iters=1000, tol=1e-6, level_iters=1, coarsest_iters=10, sync_stride=1, pure_neumann=False,
                  one_over_alpha=1.0, prolong_coeff=1.0):
        """AMGSolver::solve restated (after amg_prepare): b in channel 1, x to channel 0."""
        rel = C.c_double()
        it = oracle_lib().ocx_amg_solve(self.h, prec, max_iters, tol, level_iters, coarsest_iters, sync_stride, int(pure_neumann),
                                        one_over_alpha, prolong_coeff, C.byref(rel))
        return it, rel.value


def set_threads(n: int):
    oracle_lib().ocx_set_threads(n)


def num_threads() -> int:
    return oracle_lib().ocx_num_threads()


# ================================================================================ reference harness
_RLIB = None


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_lib():
    global _RLIB
    if _RLIB is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (oracle/build_ref.sh needs the reference tree)")
        L = C.CDLL(str(REF_LIB))
        protos = {
            "ref_device_ok": (C.c_int, []),
            "ref_create": (P, [C.c_int, C.POINTER(C.c_uint32), C.c_double]),
            "ref_destroy": (None, [P]),
            "ref_set_tile": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ref_compress_sync_spawn": (None, [P]),
            "ref_iterative_refine": (None, [P, C.POINTER(u8p), C.POINTER(C.c_int), C.c_int]),
            "ref_grid": (P, [P]),
            "ref_num_tiles": (C.c_int, [P]),
            "ref_max_level": (C.c_int, [P]),
            "ref_tiles": (None, [P, i32p]),
            "ref_slots": (None, [P, i32p]),
            "ref_set_ctypes": (None, [P, u8p]),
            "ref_get_ctypes": (None, [P, u8p]),
            "ref_calc_cell_types": (None, [P]),
            "ref_calc_neighbors": (None, [P]),
            "ref_neighbors": (None, [P, i32p]),
            "ref_set_channel": (None, [P, C.c_int, f32p]),
            "ref_get_channel": (None, [P, C.c_int, f32p]),
            "ref_rhs": (None, [P]),
            "ref_add_gradient": (None, [P, C.c_int, C.c_int]),
            "ref_full_lap": (None, [P, C.c_int, C.c_int]),
            "ref_full_lap_ex": (None, [P, C.c_int, C.c_int, C.c_int]),
            "ref_lap_same_level": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ref_gs_sweep": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ref_residual_restrict": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ref_prolongate": (None, [P, C.c_int, C.c_int, C.c_int]),
            "ref_vcycle": (None, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "ref_dot": (C.c_double, [P, C.c_int, C.c_int]),
            "ref_solve": (C.c_int, [P, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, f64p, f64p]),
            "ref_damped_jacobi": (C.c_int, [P, C.c_int, C.c_double, C.c_float, f64p]),
            "ref_last_error": (C.c_int, []),
            "ref_tile_layout": (None, [C.POINTER(C.c_longlong)]),
            "ref_refine_one_step": (None, [P, C.POINTER(u8p), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
            "ref_spawn_ghosts": (None, [P]),
            "ref_coarsen_step": (None, [P, C.POINTER(u8p), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
            "ref_statuses": (None, [P, i32p]),
            "ref_write_holder": (C.c_int, [P, C.c_int, C.c_char_p]),
            "ref_read_holder": (P, [C.c_char_p, C.c_int, C.POINTER(C.c_uint32)]),
        }
        for k, (r, a) in protos.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _RLIB = L
    return _RLIB


_RDLIB = None


def ref_dropin_lib():
    """oracle/_ref/libcirrus_ref_dropin.so (loads libcirrus_ref.so and the product library)."""
    global _RDLIB
    if _RDLIB is None:
        if not REF_DROPIN_LIB.exists():
            raise FileNotFoundError(f"{REF_DROPIN_LIB} not built (oracle/build_ref.sh)")
        ref_lib()
        L = C.CDLL(str(REF_DROPIN_LIB))
        protos = {
            "refdrop_solve": (C.c_int, [P, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, f64p, f64p]),
            "refdrop_damped_jacobi": (C.c_int, [P, C.c_int, C.c_double, C.c_float, f64p]),
            "refdrop_amg_solve": (C.c_int, [P, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, f64p]),
            "refdrop_autotune": (C.c_int, [P]),
            "refdrop_bound_grids": (C.c_int, []),
            "refdrop_release_all": (None, []),
        }
        for k, (r, a) in protos.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _RDLIB = L
    return _RDLIB


def ref_tile_layout() -> dict:
    """sizeof / offsets of the reference's PoissonTile<float> as compiled (no GPU needed)."""
    a = (C.c_longlong * 11)()
    ref_lib().ref_tile_layout(a)
    keys = ["sizeof_tile", "data", "neighbors", "cell_type", "interest", "locked", "status", "serial", "sizeof_info",
            "sizeof_T", "chnlsize"]
    return dict(zip(keys, list(a)))


class RefHarness:
    """The reference's HADeviceGrid driven through its own functions (GPU)."""

    @classmethod
    def from_holder(cls, path, log2_hash):
        """A reference grid read from a tile-holder file (its reader, setTilesFromHolder,
        compressHost, syncHostAndDevice)."""
        arr = (C.c_uint32 * len(log2_hash))(*log2_hash)
        h = ref_lib().ref_read_holder(str(path).encode(), len(log2_hash), arr)
        if not h:
            raise RuntimeError(f"reference could not read holder {path}")
        self = cls.__new__(cls)
        self.num_layers = len(log2_hash)
        self.h = h
        self.n = ref_lib().ref_num_tiles(h)
        return self

    @classmethod
    def roots(cls, w):
        """A reference grid holding only the workload's root tiles, compressed, synced and with
        ghosts spawned (src/FluidEuler.h:437-447), not yet refined."""
        L = ref_lib()
        self = cls.__new__(cls)
        self.num_layers = len(w.log2_hash)
        arr = (C.c_uint32 * self.num_layers)(*w.log2_hash)
        self.h = L.ref_create(self.num_layers, arr, w.h0)
        for r in w.roots:
            L.ref_set_tile(self.h, 0, r[0], r[1], r[2], 1)
        L.ref_compress_sync_spawn(self.h)
        self.n = L.ref_num_tiles(self.h)
        return self

    def refine_one_step(self, masks):
        keep, ptrs, dims = _mask_args(masks, self.num_layers)
        out = (C.c_int * self.num_layers)()
        ref_lib().ref_refine_one_step(self.h, ptrs, dims, self.num_layers, out)
        del keep
        self.n = ref_lib().ref_num_tiles(self.h)
        return list(out)

    def spawn_ghosts(self):
        ref_lib().ref_spawn_ghosts(self.h)
        self.n = ref_lib().ref_num_tiles(self.h)

    def coarsen_step(self, masks):
        keep, ptrs, dims = _mask_args(masks, self.num_layers)
        out = (C.c_int * self.num_layers)()
        ref_lib().ref_coarsen_step(self.h, ptrs, dims, self.num_layers, out)
        del keep
        self.n = ref_lib().ref_num_tiles(self.h)
        return list(out)

    def statuses(self):
        out = np.empty(self.n, dtype=np.int32)
        ref_lib().ref_statuses(self.h, _p(out, C.c_int32))
        return out

    def write_holder(self, path, tile_types=7):
        """getHostTileHolder(tile_types) written with the reference's file layout."""
        if ref_lib().ref_write_holder(self.h, int(tile_types), str(path).encode()) != 0:
            raise RuntimeError(f"reference could not write holder {path}")

    def __init__(self, w):
        L = ref_lib()
        self.num_layers = len(w.log2_hash)
        arr = (C.c_uint32 * self.num_layers)(*w.log2_hash)
        self.h = L.ref_create(self.num_layers, arr, w.h0)
        for r in w.roots:
            L.ref_set_tile(self.h, 0, r[0], r[1], r[2], 1)
        L.ref_compress_sync_spawn(self.h)
        keep, ptrs, dims = _mask_args(w.masks, self.num_layers)
        L.ref_iterative_refine(self.h, ptrs, dims, self.num_layers)
        del keep
        self.n = L.ref_num_tiles(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            ref_lib().ref_destroy(self.h)
            self.h = None

    def tiles(self):
        out = np.empty((self.n, 5), dtype=np.int32)
        ref_lib().ref_tiles(self.h, _p(out, C.c_int32))
        return out

    def slots(self):
        out = np.empty(self.n, dtype=np.int32)
        ref_lib().ref_slots(self.h, _p(out, C.c_int32))
        return out

    def set_ctypes(self, ct):
        a = np.ascontiguousarray(ct, dtype=np.uint8).reshape(self.n * 512)
        ref_lib().ref_set_ctypes(self.h, _p(a, C.c_uint8))

    def ctypes(self):
        out = np.empty((self.n, 512), dtype=np.uint8)
        ref_lib().ref_get_ctypes(self.h, _p(out, C.c_uint8))
        return out

    def calc_cell_types(self):
        ref_lib().ref_calc_cell_types(self.h)

    def calc_neighbors(self):
        ref_lib().ref_calc_neighbors(self.h)

    def neighbors(self):
        out = np.empty((self.n, 6), dtype=np.int32)
        ref_lib().ref_neighbors(self.h, _p(out, C.c_int32))
        return out

    def set_channel(self, c, data):
        a = np.ascontiguousarray(data, dtype=np.float32).reshape(self.n * 512)
        ref_lib().ref_set_channel(self.h, c, _p(a, C.c_float))

    def get_channel(self, c):
        out = np.empty((self.n, 512), dtype=np.float32)
        ref_lib().ref_get_channel(self.h, c, _p(out, C.c_float))
        return out

    def rhs(self, velocity):
        for a in range(3):
            self.set_channel(6 + a, velocity[a])
        ref_lib().ref_rhs(self.h)
        return self.get_channel(1)

    def add_gradient(self, p, velocity):
        """The reference's AddGradientToFaceCenters(grid, 0, 6): returns (p channel, u, v, w)."""
        self.set_channel(0, p)
        for a in range(3):
            self.set_channel(6 + a, velocity[a])
        ref_lib().ref_add_gradient(self.h, 0, 6)
        return self.get_channel(0), [self.get_channel(6 + a) for a in range(3)]

    def full_lap(self, xc, yc):
        ref_lib().ref_full_lap(self.h, xc, yc)

    def full_lap_ex(self, xc, yc, calc_diag):
        ref_lib().ref_full_lap_ex(self.h, xc, yc, int(calc_diag))

    def lap_same_level(self, tile_level, subtree_level, types, xc, yc, calc_diag=False):
        ref_lib().ref_lap_same_level(self.h, tile_level, subtree_level, types, xc, yc, int(calc_diag))

    def gs_sweep(self, level, xc, rc, color):
        ref_lib().ref_gs_sweep(self.h, level, xc, rc, color)

    def residual_restrict(self, level, xc, rhsc, coarsec):
        ref_lib().ref_residual_restrict(self.h, level, xc, rhsc, coarsec)

    def prolongate(self, level, cxc, fxc):
        ref_lib().ref_prolongate(self.h, level, cxc, fxc)

    def vcycle(self, xc=4, fc=1, rhsc=3, level_iters=1, coarsest_iters=10):
        ref_lib().ref_vcycle(self.h, xc, fc, rhsc, level_iters, coarsest_iters)

    def dot(self, a, b):
        return ref_lib().ref_dot(self.h, a, b)

    def solve(self, max_iters=1000, tol=1e-6, level_iters=1, coarsest_iters=10, sync_stride=1, pure_neumann=False):
        rel = C.c_double()
        ms = C.c_double()
        it = ref_lib().ref_solve(self.h, max_iters, tol, level_iters, coarsest_iters, sync_stride, int(pure_neumann),
                                 C.byref(rel), C.byref(ms))
        return it, rel.value, ms.value

    def damped_jacobi(self, max_iters=10, tol=1e-6, omega=1.0):
        """The reference's GMGSolver::dampedJacobiSolve: returns (iterations, relative residual)."""
        rel = C.c_double()
        it = ref_lib().ref_damped_jacobi(self.h, max_iters, tol, omega, C.byref(rel))
        return it, rel.value

    def solve_dropin(self, max_iters=1000, tol=1e-6, level_iters=1, coarsest_iters=10, sync_stride=1, pure_neumann=False):
        """GMGSolver::solve through the product's drop-in header on this reference grid, with a
        fresh solver object per call as FluidEuler::project constructs one: (iterations,
        relative residual, host-clock milliseconds of the call)."""
        rel = C.c_double()
        ms = C.c_double()
        it = ref_dropin_lib().refdrop_solve(self.h, max_iters, tol, level_iters, coarsest_iters, sync_stride, int(pure_neumann),
                                            C.byref(rel), C.byref(ms))
        if it < 0:
            raise RuntimeError("drop-in solve failed")
        return it, rel.value, ms.value

    def autotune_dropin(self):
        """cirrus_dropin::autotune on this reference grid (tunes the bound pool's launch shapes)."""
        if ref_dropin_lib().refdrop_autotune(self.h) != 0:
            raise RuntimeError("drop-in autotune failed")

    def amg_solve_dropin(self, prepare=True, max_iters=1000, tol=1e-6, level_iters=1, coarsest_iters=10, sync_stride=1,
                         pure_neumann=False):
        """AMGSolver through the product's drop-in header on this reference grid (fresh object;
        prepareTypesAndCoeffs first when `prepare`): (iterations, relative residual), or None when
        the drop-in raised (e.g. a solve without preparation for the bound pool)."""
        rel = C.c_double()
        it = ref_dropin_lib().refdrop_amg_solve(self.h, int(prepare), max_iters, tol, level_iters, coarsest_iters, sync_stride,
                                                int(pure_neumann), C.byref(rel))
        return None if it < 0 else (it, rel.value)

    def damped_jacobi_dropin(self, max_iters=10, tol=1e-6, omega=1.0):
        """The same call through the product's drop-in header on this reference grid."""
        rel = C.c_double()
        it = ref_dropin_lib().refdrop_damped_jacobi(self.h, max_iters, tol, omega, C.byref(rel))
        if it < 0:
            raise RuntimeError("drop-in damped Jacobi failed")
        return it, rel.value
