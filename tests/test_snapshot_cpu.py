"""The reference's snapshot format for the liquid's parts, on the CPU: a
world saved and loaded again holds the same buffers, a reference-shaped
snapshot (current cells in the second buffer, parts the liquid doesn't
use) loads and saves back intact, bad files are refused as the reference
refuses them, and a world loaded from a snapshot steps on (the oracle) as
the world it was saved from does, tiling parity included."""
import gzip
import json
import struct

import numpy as np
import pytest

from worldinagrain_b200 import abi, snapshot
from worldinagrain_b200 import world as W

from .common import compare_worlds, params


def _world():
    return W.small_world(48, 40, seed=5, kind="obstacles")


def test_round_trip_keeps_every_buffer_and_the_state():
    w = _world()
    w.sorted[0] = 7
    w.counters[:5] = [1, 2, 3, 4, 5]
    data = snapshot.save(w, state={"frameNo": 12, "shiftedFirst": True, "fluidCycles": 9})
    header, parts = snapshot.read(data)
    assert header["format"] == 1 and header["width"] == 48 and header["height"] == 40
    assert header["state"] == {"frameNo": 12, "shiftedFirst": True, "fluidCycles": 9, "cur": 0}
    assert [p["name"] for p in header["parts"]][:2] == ["cells0", "cells1"]
    got = snapshot.world_from(header, parts)
    assert not compare_worlds(got, w)
    assert got.cap == w.cap and got.snapshot_state["frameNo"] == 12


def test_reference_shaped_snapshot_loads_and_saves_back():
    w = _world()
    stale = np.full_like(w.cells, 0xDEADBEEF)
    air = np.arange(100, dtype=np.uint32)
    parts = {"cells0": stale, "cells1": w.cells, "air": air, "particles0": w.sorted, "particles1": w.parts,
             "counters": w.counters, "field": w.field, "blocks": w.blocks}
    header = {"format": 1, "width": 48, "height": 40, "elements": [0, 1, 2, 3, 4],
              "state": {"cur": 1, "frameNo": 3, "shiftedFirst": False}}
    got = snapshot.load(snapshot.write(header, parts))
    assert np.array_equal(got.cells, w.cells)          # cells1: the current one
    assert np.array_equal(got.cg, np.zeros_like(w.cg))  # fluidCg not kept: zero
    again_h, again = snapshot.read(snapshot.save(got))
    assert np.array_equal(again["air"].view(np.uint32), air)  # outside the liquid: kept as it was
    assert np.array_equal(again["cells0"].view(np.uint32), w.cells)
    assert np.array_equal(again["cells1"].view(np.uint32), stale)
    assert again_h["state"]["cur"] == 0 and again_h["elements"] == [0, 1, 2, 3, 4]


def _raw(header, body=b""):
    head = json.dumps(header).encode()
    return gzip.compress(b"SANDSNAP" + struct.pack("<I", len(head)) + head + b"\0" * (-len(head) % 4) + body)


def test_bad_files_are_refused():
    w = _world()
    with pytest.raises(ValueError, match="not a snapshot"):
        snapshot.read(b"plainly not gzip")
    with pytest.raises(ValueError, match="not a snapshot"):
        snapshot.read(gzip.compress(b"SANDSNAQ" + b"\0" * 8))
    with pytest.raises(ValueError, match="format 2"):
        snapshot.read(_raw({"format": 2, "parts": []}))
    with pytest.raises(ValueError, match="cut short"):
        snapshot.read(_raw({"format": 1, "parts": [{"name": "x", "bytes": 64}]}, b"\0" * 8))
    header, parts = snapshot.read(snapshot.save(w))
    parts["field"] = parts["field"][:-4]
    with pytest.raises(ValueError, match="field"):
        snapshot.world_from(header, parts)
    del parts["counters"]
    with pytest.raises(ValueError, match="counters"):
        snapshot.world_from(header, parts)


def test_loaded_world_steps_on_as_the_saved_one():
    from oracle.oracle import Oracle
    base = _world()
    full = base.copy()
    o = Oracle(full, W.element_table())
    for s in range(1, 4):
        o.step(params(full, s))
    part = base.copy()
    a = Oracle(part, W.element_table())
    for s in range(1, 3):
        a.step(params(part, s))
    data = snapshot.save(part, state={"frameNo": 2, "shiftedFirst": bool(a.shifted.value)})
    loaded = snapshot.load(data)
    b = Oracle(loaded, W.element_table())
    b.step(params(loaded, 3), flags=snapshot.step_flags(loaded))
    d = compare_worlds(loaded, full, region_links=True)
    assert not d, "; ".join(d)
    assert snapshot.step_flags(loaded) & abi.STEP_SHIFTED_SET
