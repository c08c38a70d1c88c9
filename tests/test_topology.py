"""Host topology: the product's builder against the oracle restatement and against the
reference's own construction (golden fixtures from the reference build).  Integer work,
compared bit for bit: tile order (hash-slot order, level-major), tile types, hash slots,
neighbour tables and cell types."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden_npz
from cirrus_b200 import workloads as W
from oracle import oracle as O

SMALL = ["uniform32_small", "sphere64_small", "sphere64_neumann_small", "ring64_small"]
FULL = ["uniform128", "sphere256", "sphere256_neumann", "ring512"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", SMALL)
def test_product_matches_oracle_small(name, built_cache):
    b = built_cache(name)
    w = b.workload
    ot = O.oracle_topology(w)
    assert np.array_equal(ot.tiles(), b.tiles)
    assert np.array_equal(ot.slots(), b.topology.hash_slots())
    f = O.CpuOracle(b.tiles)
    assert np.array_equal(f.neighbors(), b.nbr6)
    f.set_ctypes(W.leaf_cell_types(w, b.tiles, b.nbr6))
    f.calc_cell_types()
    assert np.array_equal(f.ctypes(), b.ctypes)


@pytest.mark.slow
@pytest.mark.parametrize("name", FULL)
def test_product_matches_oracle_full(name, built_cache):
    b = built_cache(name)
    ot = O.oracle_topology(b.workload)
    assert np.array_equal(ot.tiles(), b.tiles)
    assert np.array_equal(ot.slots(), b.topology.hash_slots())


@pytest.mark.parametrize("name", SMALL)
def test_oracle_and_product_match_reference_small(name, built_cache):
    g = golden_npz(name)
    b = built_cache(name)
    ot = O.oracle_topology(b.workload)
    assert np.array_equal(g["tiles"], b.tiles)
    assert np.array_equal(g["tiles"], ot.tiles())
    assert np.array_equal(g["slots"], b.topology.hash_slots())
    assert np.array_equal(g["nbr"], b.nbr6)
    assert np.array_equal(g["ctypes"], b.ctypes)


@pytest.mark.parametrize("name", FULL)
def test_product_matches_reference_digests_full(name, built_cache, golden_summary):
    if name not in golden_summary:
        pytest.skip("no reference summary for this workload")
    d = golden_summary[name]["digests"]
    b = built_cache(name)
    assert digest(b.tiles) == d["tiles"]
    assert digest(b.topology.hash_slots()) == d["slots"]
    assert digest(b.nbr6) == d["nbr"]
    assert digest(b.ctypes) == d["ctypes"]
    assert golden_summary[name]["dof"] == b.dof()


def test_uniform128_shape():
    b = W.build(W.make("uniform128"))
    c = b.counts()
    assert c["leaf"] == 4096 and c["nonleaf"] == 1 + 8 + 64 + 512 and c["ghost"] == 0
    assert c["dof"] == 126 ** 3


def test_two_to_one_balance_and_ghost_parents(built_cache):
    """Every GHOST tile's parent is a LEAF; face-adjacent LEAF tiles differ by at most one level."""
    b = built_cache("sphere64_small")
    t = b.tiles
    key = {(int(l), int(x), int(y), int(z)): i for i, (l, x, y, z, _) in enumerate(t)}
    for i, (l, x, y, z, ty) in enumerate(t):
        if ty == W.GHOST:
            p = key.get((l - 1, x >> 1, y >> 1, z >> 1))
            assert p is not None and t[p, 4] == W.LEAF
    # 2:1 face balance: across each face of a LEAF tile, a NONLEAF neighbour's four children on
    # the shared face are LEAF tiles (never refined further)
    for i, (l, x, y, z, ty) in enumerate(t):
        if ty != W.LEAF:
            continue
        for axis in range(3):
            for sgn in (-1, 1):
                n = [int(x), int(y), int(z)]
                n[axis] += sgn
                nb = key.get((int(l), *n))
                if nb is None or t[nb, 4] != W.NONLEAF:
                    continue
                for o in range(8):
                    off = [o & 1, (o >> 1) & 1, (o >> 2) & 1]
                    if off[axis] != (1 if sgn < 0 else 0):
                        continue
                    ch = key.get((int(l) + 1, n[0] * 2 + off[0], n[1] * 2 + off[1], n[2] * 2 + off[2]))
                    assert ch is not None and t[ch, 4] == W.LEAF


def test_refine_callback_equals_masks():
    """IterativeRefine through a level-target callback builds the same tree as through masks."""
    from cirrus_b200 import Topology

    w = W.make("sphere64_small")
    t1 = Topology(w.h0, w.log2_hash)
    t1.set_tile(0, (0, 0, 0), W.LEAF)
    t1.compress()
    t1.spawn_ghost_tiles()
    t1.iterative_refine(masks=w.masks)

    def target(l, x, y, z):
        m = w.masks[l] if l < len(w.masks) else None
        if m is None or min(x, y, z) < 0 or x >= m.shape[0] or y >= m.shape[1] or z >= m.shape[2]:
            return l
        return l + 1 if m[x, y, z] else l
    t2 = Topology(w.h0, w.log2_hash)
    t2.set_tile(0, (0, 0, 0), W.LEAF)
    t2.compress()
    t2.spawn_ghost_tiles()
    t2.iterative_refine(level_target=target)
    assert np.array_equal(t1.tiles(), t2.tiles())


def test_hash_table_full_is_reported():
    from cirrus_b200 import Topology, CirrusError

    t = Topology(1 / 8, (2, 2))
    for i in range(4):
        t.set_tile(0, (i, 0, 0), W.LEAF)
    with pytest.raises(CirrusError):
        t.set_tile(0, (9, 9, 9), W.LEAF)
