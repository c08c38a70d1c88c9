"""The C-ABI library loads and exports every entry point that include/*.h declares (CPU only:
no compute call is made here)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

from conftest import ROOT


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(cirrus_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_functions():
    names = declared_functions()
    assert "cirrus_gmg_solve" in names and "cirrus_topology_create" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    from cirrus_b200 import _native

    lib = _native.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_header():
    from cirrus_b200 import _native

    assert set(declared_functions()) == set(_native.exported_symbols())


def test_status_strings_and_defaults():
    from cirrus_b200 import _native

    lib = _native.lib()
    assert lib.cirrus_status_string(0) == b"ok"
    assert b"sm_100a" in lib.cirrus_version()
    p = _native.SolveParams()
    lib.cirrus_solve_params_default(C.byref(p))
    # the reference call site: solve(grid, false, 1000, 1e-6, 1, 10, 1, pure_neumann)
    assert (p.max_iters, p.relative_tolerance, p.level_iters, p.coarsest_iters, p.sync_stride) == (1000, 1e-6, 1, 10, 1)
    assert p.one_over_alpha == 1.0 and p.prolong_coeff == 1.0


def test_invalid_arguments_are_rejected_without_a_device():
    from cirrus_b200 import _native

    lib = _native.lib()
    h = C.c_void_p()
    bad = (C.c_uint32 * 1)(40)
    assert lib.cirrus_topology_create(1, bad, 0.125, C.byref(h)) == 1
    assert lib.cirrus_topology_create(0, bad, 0.125, C.byref(h)) == 1
    assert lib.cirrus_gmg_solve(None, None, None, None) == 1
    assert lib.cirrus_grid_create(None, C.byref(h)) == 1
    it, rel = C.c_int(), C.c_double()
    assert lib.cirrus_damped_jacobi_solve(None, 10, 1e-6, 1.0, None, C.byref(it), C.byref(rel)) == 1
    assert lib.cirrus_full_negative_laplacian_ex(None, 2, 3, 1, None) == 1
    assert lib.cirrus_negative_laplacian_same_level(None, -1, -1, 5, 2, 3, 0, None) == 1
    assert lib.cirrus_gmg_solve_host_submit(None, None, None, None, None) == 1
    assert lib.cirrus_gmg_solve_host_wait(None, None) == 1


def test_library_is_built_for_sm100a():
    from cirrus_b200 import build

    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)
    assert Path(build.LIB).exists()
