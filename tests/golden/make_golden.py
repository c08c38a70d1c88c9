"""Generate the golden fixtures of tests/golden/ by running the reference's own CUDA build.

The reference (wang-mengdi/Cirrus) ships no tests, fixtures or golden vectors for the Poisson
path, so its results are pinned by running its unmodified sources (compiled by
oracle/build_ref.sh into oracle/_ref/libcirrus_ref.so) on a B200 through oracle/ref_harness.cu:
  * topology: IterativeRefine + SpawnGhostTiles + CalcCellTypesFromLeafs + CalculateNeighborTiles
    (tiles in dAllTiles order, hash slots, neighbour table, cell types);
  * right-hand side: face clearing, PropagateToChildren, VelocityVolumeDivergenceOnLeafs;
  * operators: FullNegativeLaplacian of b, one V-cycle of b;
  * GMGSolver::solve(grid, false, 1000, 1e-6, 1, 10, 1, pure_neumann) as FluidEuler::project
    calls it (iterations, relative residual, pressure).
Small workloads are stored whole (compressed .npz); full-size ones as SHA-256 digests of the
integer arrays plus the solve summary and a strided sample of the pressure.

Usage (on a GPU machine, from the repository root):  python tests/golden/make_golden.py OUTDIR
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from cirrus_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

SMALL = ["uniform32_small", "sphere64_small", "sphere64_neumann_small", "ring64_small"]
FULL = ["uniform128", "sphere256", "sphere256_neumann", "ring512"]
SAMPLE_STRIDE = 97


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run(name: str, full: bool, out: Path) -> dict:
    w = W.make(name)
    t0 = time.time()
    ref = O.RefHarness(w)
    tiles = ref.tiles()
    slots = ref.slots()
    ref.calc_neighbors()
    nbr = ref.neighbors()
    leaf_ct = W.leaf_cell_types(w, tiles, nbr)
    ref.set_ctypes(leaf_ct)
    ref.calc_cell_types()
    ref.calc_neighbors()
    ctypes = ref.ctypes()
    vel = W.face_velocity(tiles, w.seed)
    b = ref.rhs(vel)
    # FullNegativeLaplacian of b (channel 2 -> 3)
    ref.set_channel(2, b)
    ref.full_lap(2, 3)
    ap = ref.get_channel(3)
    # one V-cycle of b (z <- M^-1 b)
    ref.set_channel(1, b)
    ref.vcycle(4, 1, 3, 1, 10)
    z = ref.get_channel(4)
    # the solve as FluidEuler::project calls it
    ref.set_channel(1, b)
    ref.set_channel(0, np.zeros_like(b))
    iters, rel, ms = ref.solve(1000, 1e-6, 1, 10, 1, w.pure_neumann)
    x = ref.get_channel(0)
    leaf = (tiles[:, 4] & 1) != 0
    summary = {
        "workload": name, "tiles": int(tiles.shape[0]), "dof": int(((ctypes[leaf] & 2) != 0).sum()),
        "iters": int(iters), "rel_residual": float(rel), "solve_ms": float(ms),
        "x_norm": float(np.sqrt((x[leaf].astype(np.float64) ** 2).sum())),
        "b_norm": float(np.sqrt((b[leaf].astype(np.float64) ** 2).sum())),
        "digests": {"tiles": digest(tiles), "slots": digest(slots), "nbr": digest(nbr), "ctypes": digest(ctypes),
                    "b": digest(b), "ap": digest(ap)},
        "seconds": time.time() - t0,
    }
    if full:
        idx = np.arange(0, x.size, SAMPLE_STRIDE)
        np.savez_compressed(out / f"{name}.npz", x_sample=x.reshape(-1)[idx], z_sample=z.reshape(-1)[idx],
                            sample_stride=np.int64(SAMPLE_STRIDE))
    else:
        np.savez_compressed(out / f"{name}.npz", tiles=tiles, slots=slots, nbr=nbr, ctypes=ctypes, b=b, ap=ap, z=z, x=x,
                            iters=np.int64(iters), rel=np.float64(rel))
    return summary


def main():
    out = Path(sys.argv[1] if len(sys.argv) > 1 else ROOT / "tests" / "golden")
    out.mkdir(parents=True, exist_ok=True)
    names = sys.argv[2:] or (SMALL + FULL)
    summaries = {}
    for name in names:
        s = run(name, name in FULL, out)
        summaries[name] = s
        print(json.dumps({k: v for k, v in s.items() if k != "digests"}), flush=True)
    path = out / "reference_summary.json"
    old = json.loads(path.read_text()) if path.exists() else {}
    old.update(summaries)
    path.write_text(json.dumps(old, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
