"""Tile-holder files (the reference's IOFunc::WriteHAHostTileHolderToFile format,
src/PoissonIOFunc.cu:38-121) on the CPU: the record layout against the reference's compiled
PoissonTile<float>, files encoded here independently (numpy, from those offsets) read by the
product, the product's writer reproducing them byte for byte, the setTilesFromHolder +
compressHost topology, and refusal of damaged files."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from cirrus_b200 import CirrusError, Holder
from oracle import oracle as O

LAYOUT = {"sizeof_tile": 33104, "data": 0, "neighbors": 32384, "cell_type": 32576, "interest": 33088, "locked": 33089,
          "status": 33092, "serial": 33096, "sizeof_info": 32, "sizeof_T": 4, "chnlsize": 736}


def encode_holder(h0, num_layers, max_level, tiles5, channels, ctypes, neighbor_junk=True):
    """A holder file built byte by byte from the layout: tiles5 (n, 5) in level-major order,
    channels {c: (n, 512) float32}, ctypes (n, 512) uint8."""
    n = tiles5.shape[0]
    rec = np.zeros((n, LAYOUT["sizeof_tile"]), dtype=np.uint8)
    for c, a in channels.items():
        off = LAYOUT["data"] + c * LAYOUT["chnlsize"] * 4
        rec[:, off:off + 2048] = np.ascontiguousarray(a, dtype=np.float32).view(np.uint8).reshape(n, 2048)
    if neighbor_junk:  # pointers of the writing process: arbitrary bytes the reader must ignore
        rec[:, LAYOUT["neighbors"]:LAYOUT["neighbors"] + 192] = 0xAB
    rec[:, LAYOUT["cell_type"]:LAYOUT["cell_type"] + 512] = ctypes
    out = bytearray(struct.pack("<fiiQ", h0, num_layers, max_level, n))
    out += rec.tobytes()
    out += struct.pack("<Q", num_layers)
    for l in range(num_layers):
        idx = np.flatnonzero(tiles5[:, 0] == l)
        out += struct.pack("<Q", idx.size)
        for i in idx:
            out += struct.pack("<iiiiBq", int(tiles5[i, 1]), int(tiles5[i, 2]), int(tiles5[i, 3]), l, int(tiles5[i, 4]), int(i))
    return bytes(out)


def test_record_layout_matches_the_reference_build():
    if not O.REF_LIB.exists():
        pytest.skip("reference build oracle/_ref/libcirrus_ref.so not present")
    assert O.ref_tile_layout() == LAYOUT


@pytest.mark.parametrize("name", ["uniform32_small", "ring64_small"])
def test_read_write_round_trip_and_topology(tmp_path, built_cache, name):
    b = built_cache(name)
    t5 = b.tiles
    rng = np.random.default_rng(3)
    chans = {c: rng.standard_normal((b.n, 512)).astype(np.float32) for c in (0, 1, 6, 9)}
    blob = encode_holder(np.float32(b.workload.h0), b.workload.num_layers, int(t5[:, 0].max()), t5, chans, b.ctypes)
    p = tmp_path / "a.bin"
    p.write_bytes(blob)
    h = Holder.read(p)
    info = h.info()
    assert info["num_tiles"] == b.n and info["num_layers"] == b.workload.num_layers
    assert info["max_level"] == int(t5[:, 0].max()) and info["h0"] == float(np.float32(b.workload.h0))
    assert np.array_equal(h.tiles(), t5)
    assert np.array_equal(h.cell_types(), b.ctypes)
    for c in range(11):
        want = chans.get(c, np.zeros((b.n, 512), np.float32))
        assert np.array_equal(h.channel(c).view(np.uint32), want.view(np.uint32)), c
    # the product's writer reproduces the file (neighbour bytes aside, which it writes as zeros)
    q = tmp_path / "b.bin"
    h.write(q)
    again = encode_holder(np.float32(b.workload.h0), b.workload.num_layers, int(t5[:, 0].max()), t5, chans, b.ctypes,
                          neighbor_junk=False)
    written = q.read_bytes()
    assert len(written) == len(blob)
    # records copied as read: the junk neighbour bytes survive a read/write cycle unchanged
    assert written == blob
    assert len(again) == len(blob)
    # setTilesFromHolder + compressHost: the same tiles, hash order and cell types
    topo, order = h.to_topology(b.workload.log2_hash)
    assert np.array_equal(topo.tiles(), t5)
    assert np.array_equal(order, np.arange(b.n))
    assert np.array_equal(topo.hash_slots(), b.topology.hash_slots())
    assert np.array_equal(topo.cell_types(), b.ctypes)


def test_damaged_files_are_refused(tmp_path, built_cache):
    b = built_cache("uniform32_small")
    blob = encode_holder(np.float32(0.125), 10, 2, b.tiles, {}, b.ctypes)
    for cut in (3, 20, 20 + 33104 * 5, len(blob) - 7):
        p = tmp_path / f"cut{cut}.bin"
        p.write_bytes(blob[:cut])
        with pytest.raises(CirrusError):
            Holder.read(p)
    bad = bytearray(blob)
    # a tile info whose record index lies past the records
    struct.pack_into("<q", bad, len(bad) - 8, 10 ** 6)
    p = tmp_path / "bad_index.bin"
    p.write_bytes(bytes(bad))
    with pytest.raises(CirrusError):
        Holder.read(p)
    with pytest.raises(CirrusError):
        Holder.read(tmp_path / "missing.bin")
    # a different layer count than the grid's hash sizes
    h = Holder.read(_write(tmp_path / "ok.bin", blob))
    with pytest.raises(CirrusError):
        h.to_topology((16, 16, 16))


def _write(p, blob):
    p.write_bytes(blob)
    return p
