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
    header = {"format": 1, "width": 48, "height": 40, "elements": [0, 1, 2, 3, 4], "gas": 2, "bodies": 1,
              "water": {"vapour20": 1.0}, "state": {"cur": 1, "frameNo": 3, "shiftedFirst": False}}
    got = snapshot.load(snapshot.write(header, parts))
    assert np.array_equal(got.cells, w.cells)          # cells1: the current one
    assert not got.cg.any()  # the CG vectors are written before they are read: not a part
    again_h, again = snapshot.read(snapshot.save(got))
    assert np.array_equal(again["air"].view(np.uint32), air)  # outside the liquid: kept as it was
    assert np.array_equal(again["cells0"].view(np.uint32), w.cells)
    assert np.array_equal(again["cells1"].view(np.uint32), stale)
    assert again_h["state"]["cur"] == 0 and again_h["elements"] == [0, 1, 2, 3, 4]
    # the header keys the other parts' loaders read, written back as loaded
    assert again_h["gas"] == 2 and again_h["bodies"] == 1 and again_h["water"] == {"vapour20": 1.0}
    with pytest.raises(ValueError, match="different set of elements"):
        snapshot.load(snapshot.write(header, parts), element_ids=[0, 1, 2, 3])


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
    # malformed headers and part lists: a ValueError, never another error
    for h, body in (({"format": 1, "parts": [{"name": "x", "bytes": -5}]}, b"\0" * 16),
                    ({"format": 1, "parts": [{"name": "x", "bytes": "4"}]}, b"\0" * 16),
                    ({"format": 1, "parts": [{"bytes": 4}]}, b"\0" * 16),
                    ({"format": 1, "parts": 5}, b""),
                    ([1, 2], b"")):
        with pytest.raises(ValueError):
            snapshot.read(_raw(h, body))
    with pytest.raises(ValueError, match="cut short"):
        snapshot.read(gzip.compress(b"SANDSNAP" + struct.pack("<I", 10 ** 9) + b"{}"))
    header, parts = snapshot.read(snapshot.save(w))
    for h in ({k: v for k, v in header.items() if k != "width"}, dict(header, height="tall"),
              dict(header, width=0), dict(header, state=[]), dict(header, state={"cur": 2})):
        with pytest.raises(ValueError):
            snapshot.world_from(h, parts)
    bad = dict(parts, field=parts["field"][:-4])
    with pytest.raises(ValueError, match="lays out field differently"):
        snapshot.world_from(header, bad)
    bad = dict(parts, cells1=parts["cells1"][:-16])  # the pair's other buffer must fit too
    with pytest.raises(ValueError, match="cells1"):
        snapshot.world_from(header, bad)
    bad = {k: v for k, v in parts.items() if k != "particles0"}
    with pytest.raises(ValueError, match="particles0"):
        snapshot.world_from(header, bad)
    other = W.World(40, 40)
    before = other.cells.copy()
    with pytest.raises(ValueError, match="48x40 world"):
        snapshot.restore(other, header, parts)
    assert np.array_equal(other.cells, before)  # nothing changed


def test_particles_laid_out_otherwise_load_empty_with_the_liquid_undrawn():
    """A snapshot whose particle buffers are of another capacity loads as
    migrateLiquid has it: no particles, counters or blocks, its liquid cells
    undrawn with the run word cleared, everything else as saved."""
    w = _world()
    from oracle.oracle import Oracle
    o = Oracle(w, W.element_table())
    for s in range(1, 3):
        o.step(params(w, s))
    header, parts = snapshot.read(snapshot.save(w))
    parts["particles0"] = parts["particles0"][:-48]
    parts["particles1"] = parts["particles1"][:-48]
    got = snapshot.world_from(header, parts)
    assert got.snapshot_migrated
    for buf in ("sorted", "parts", "counters", "blocks"):
        assert not getattr(got, buf).any(), buf
    assert np.array_equal(got.field, w.field)
    cw, gw = w.cell_view(), got.cell_view()
    liquid = (cw[..., 0] & 0xFF) == abi.WATER
    assert liquid.any() and (cw[liquid, 0] >> 28 & 4).any()
    assert not (gw[liquid, 0] >> 28 & 4).any() and not gw[liquid, 3].any()
    assert np.array_equal(gw[liquid, 0] | (4 << 28), cw[liquid, 0] | (4 << 28))
    assert np.array_equal(gw[~liquid], cw[~liquid])
    b = Oracle(got, W.element_table())
    b.step(params(got, 3), flags=snapshot.step_flags(got))
    assert got.sorted[0] >= 4 * liquid.sum() * 0.9  # the liquid seeded afresh


def test_older_blocks_and_field_are_widened_with_zeros():
    w = _world()
    w.blocks[:] = np.arange(w.blocks.size, dtype=np.uint32) + 1
    w.field[:] = np.arange(w.field.size, dtype=np.float32) + 1
    header, parts = snapshot.read(snapshot.save(w))
    B, F = w.L["block_count"], w.L["face_count"]
    at = 4 * B + 4
    blocks = parts["blocks"].view(np.uint32)
    parts["blocks"] = np.concatenate([blocks[:at], blocks[at + abi.FLUID_STATS - 4:]]).view(np.uint8)
    q = (F + 3) // 4 * 4
    f0 = w.C * 8 + F * 4 + q
    field = parts["field"].view(np.float32)
    parts["field"] = np.concatenate([field[:f0], field[f0 + q:]]).view(np.uint8)
    got = snapshot.world_from(header, parts)
    assert not got.snapshot_migrated
    want = w.blocks.copy()
    want[at:at + abi.FLUID_STATS - 4] = 0
    assert np.array_equal(got.blocks, want)
    want = w.field.copy()
    want[f0:f0 + q] = 0
    assert np.array_equal(got.field, want)


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


# ---------------------------------------------------------------- free bodies' parts

def _body_snapshot(w, bodies, header_bodies=True, motion=None, stamps=None):
    """A snapshot of w with the bodies' parts (bodyMotion, bodies) as given
    (the current layouts by default); header_bodies: whether its header says
    the bodies were kept whole (BODIES)."""
    w.snapshot_rest = {"bodyMotion": (bodies.motion if motion is None else motion).view(np.uint8),
                       "bodies": (bodies.stamps if stamps is None else stamps).view(np.uint8)}
    data = snapshot.save(w, state={"frameNo": 2})
    header, parts = snapshot.read(data)
    if not header_bodies:
        del header["bodies"]
    return header, parts


def _oracle(world, bodies):
    from oracle.oracle import Oracle
    return Oracle(world, W.body_element_table(), bodies)


def test_bodies_round_trip_and_step_on_as_saved():
    """A world with free bodies saved after two steps and loaded again holds
    the same buffers and body table, and steps on (the oracle, coupled) as
    the world it was saved from."""
    w, bodies = W.bodies_world()
    o = _oracle(w, bodies)
    flags = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS | abi.STEP_SHIFTED_SET
    for s in (1, 2):
        bodies.stamp_step(s - 1)
        o.step(params(w, s), max_cycles=64, flags=flags, tolerance=1e-6)
    snapshot.keep_bodies(w, bodies)
    header, parts = _body_snapshot(w, bodies)
    assert header["bodies"] == snapshot.BODIES
    got = snapshot.world_from(header, parts, elems=W.body_element_table())
    got_b = snapshot.bodies_from(got)
    assert got_b is not None
    assert np.array_equal(got_b.motion, bodies.motion) and np.array_equal(got_b.stamps, bodies.stamps)
    assert not compare_worlds(got, w, grid=("cells", "counters", "field", "blocks"))  # cg is no part
    got_b.swept = bodies.swept
    o2 = _oracle(got, got_b)
    bodies.stamp_step(2)
    got_b.stamp_step(2)
    o.step(params(w, 3), max_cycles=64, flags=flags, tolerance=1e-6)
    o2.step(params(got, 3), max_cycles=64, flags=flags, tolerance=1e-6)
    assert not compare_worlds(got, w)
    assert np.array_equal(got_b.motion, bodies.motion) and np.array_equal(got_b.pushes, bodies.pushes)


def test_narrow_body_tables_are_widened():
    """Body slots saved OLD_TABLE_WORDS wide are widened with zeros, the
    contacts and the liquid's words moved along (migrateTable)."""
    w, bodies = W.bodies_world()
    nb, tw, ow = abi.MAX_BODIES, abi.BODY_TABLE_WORDS, snapshot.OLD_TABLE_WORDS
    bodies.motion[nb:nb * (1 + tw)].reshape(nb, tw)[:, ow:] = 0  # what an old table could not hold
    bodies.motion[nb * (1 + tw):] = np.arange(bodies.motion.size - nb * (1 + tw), dtype=np.uint32)
    old = np.concatenate([bodies.motion[:nb], bodies.motion[nb:nb * (1 + tw)].reshape(nb, tw)[:, :ow].ravel(),
                          bodies.motion[nb * (1 + tw):]])
    header, parts = _body_snapshot(w, bodies, motion=old)
    got = snapshot.bodies_from(snapshot.world_from(header, parts, elems=W.body_element_table()))
    assert np.array_equal(got.motion, bodies.motion)


def test_swept_words_at_the_start_of_the_table_are_moved():
    """Two words a cell saved at the start of bodyMotion, from before the
    stamps moved to the end of the bodies buffer: dropped there, none at the
    end (migrateSwept)."""
    w, bodies = W.bodies_world()
    cell_words = 2 * w.C
    bodies.stamps[-cell_words:] = 0
    old_motion = np.concatenate([np.full(cell_words, 0xABCDEF, dtype=np.uint32), bodies.motion])
    header, parts = _body_snapshot(w, bodies, motion=old_motion, stamps=bodies.stamps[:-cell_words])
    got = snapshot.bodies_from(snapshot.world_from(header, parts, elems=W.body_element_table()))
    assert np.array_equal(got.motion, bodies.motion) and np.array_equal(got.stamps, bodies.stamps)


def test_bodies_not_kept_whole_let_go_of_cells_they_did_not_stamp():
    """A snapshot from before its bodies were kept whole: live bodies are
    looked at whole (PARTS), and loose cells their body did not claim in
    its last step are let go, FREE_BODY in their slot (migrateBodies); the
    liquid step then takes them as no body's."""
    w, bodies = W.bodies_world()
    nb, tw = abi.MAX_BODIES, abi.BODY_TABLE_WORDS
    frame = 5
    bodies.words(0)[abi.BW["FRAME"]] = frame
    tiles = -(-w.W // abi.BODY_TILE) * -(-w.H // abi.BODY_TILE)
    claims_at = 4 * tiles + abi.BODY_STAT_WORDS + abi.BODY_COUNTERS + nb + w.C
    cv = w.cell_view().reshape(w.C, 4)
    slot = (cv[:, 3] & 0xFFFF).astype(np.uint16).view(np.float16)
    loose = ((cv[:, 0] >> 28) & abi.FL_LOOSE) != 0
    mine = np.flatnonzero(loose & (slot == 0))
    bodies.stamps[claims_at + mine] = ((frame & 0xFFFFF) << 12) | ((2047 - 0) << 1)
    header, parts = _body_snapshot(w, bodies, header_bodies=False)
    got = snapshot.world_from(header, parts, elems=W.body_element_table())
    gslot = (got.cell_view().reshape(w.C, 4)[:, 3] & 0xFFFF).astype(np.uint16).view(np.float16)
    assert np.all(gslot[mine] == 0)
    others = np.flatnonzero(loose & (slot != 0))
    assert others.size and np.all(gslot[others] == np.float16(snapshot.FREE_BODY))
    gb = snapshot.bodies_from(got)
    flags = gb.motion[nb:nb * (1 + tw)].reshape(nb, tw)[:, abi.BW["FLAGS"]]
    live = (bodies.motion[nb:nb * (1 + tw)].reshape(nb, tw)[:, abi.BW["FLAGS"]] & abi.BF_ALIVE) != 0
    assert np.all((flags[live] & 8) != 0) and not np.any(flags[~live] & 8)
    # kept whole: nothing let go
    header, parts = _body_snapshot(w, bodies)
    kept = snapshot.world_from(header, parts, elems=W.body_element_table())
    assert np.array_equal(kept.cells, w.cells)
