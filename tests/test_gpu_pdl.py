"""Programmatic dependent launch changes no result.

The stencil, coarse-level and vector kernels read the grid's topology (tile lists, metadata,
coefficient classes, level constants, masks, chunk tables) before they wait on their predecessor,
so that those loads overlap the predecessor's tail.  Launched without the programmatic attribute
(CIRRUS_NO_PDL=1, read once per process, hence the child processes) every kernel starts only after
its predecessor has finished; both launches must give the same iterations and pressure bit for
bit.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]

CHILD = r"""
import sys
import numpy as np
from cirrus_b200 import DeviceGrid, GMGSolver, workloads as W
names = sys.argv[2].split(",")
bs = [W.build(W.make(n, 0)) for n in names]
g = DeviceGrid([b.topology for b in bs])
for i, b in enumerate(bs):
    for a in range(3):
        g.set_channel_instance(i, 6 + a, b.velocity[a])
g.projection_rhs()
s = GMGSolver()
res = s.solve_batch(g)
assert all(r.status == 0 for r in s.last_results)
xs = {f"x{i}": g.get_channel_instance(i, 0) for i in range(len(bs))}
np.savez(sys.argv[1], iters=np.array([r[0] for r in res]), rel=np.array([r[1] for r in res]), **xs)
g.close()
"""


@pytest.mark.parametrize("names", [["sphere64_small", "ring64_small"], ["ring512", "ring512"]])
def test_launches_without_programmatic_dependence_give_the_same_bits(tmp_path, names):
    out = {}
    for mode in ("pdl", "plain"):
        env = dict(os.environ)
        env.pop("CIRRUS_NO_PDL", None)
        if mode == "plain":
            env["CIRRUS_NO_PDL"] = "1"
        path = tmp_path / f"{mode}.npz"
        subprocess.run([sys.executable, "-c", CHILD, str(path), ",".join(names)], env=env, cwd=REPO, check=True, timeout=900)
        out[mode] = np.load(path)
    a, b = out["pdl"], out["plain"]
    assert np.array_equal(a["iters"], b["iters"])
    assert np.array_equal(a["rel"].view(np.uint64), b["rel"].view(np.uint64))
    for i in range(len(names)):
        assert np.array_equal(a[f"x{i}"].view(np.uint32), b[f"x{i}"].view(np.uint32)), i
