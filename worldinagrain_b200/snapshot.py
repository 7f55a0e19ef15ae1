"""The reference's snapshot format (js/snapshot.js), for the liquid's parts:
worlds saved by the reference load into this library's resident buffers,
and worlds stepped here save in a form the reference reads back.

A snapshot is gzipped (js/snapshot.js:4-8, :127-156, :163-189):

- MAGIC ("SANDSNAP");
- the header's length in bytes (u32, little-endian);
- the header: JSON with the format (1), the world's width and height, the
  elements by id, the simulation's state (Simulation.snapshotState,
  js/sim.js:1445-1465) and each part's name and size;
- each part's bytes in the header's order, each padded to 4.

The parts are the GPU buffers that carry over from one step to the next
(Simulation.snapshotParts, js/sim.js:1429-1438: what js/passes.js:161-182
finds read before it is written), a pair named name0 and name1. The
liquid's are:

- cells0 and cells1, the state's `cur` the one the next step reads;
- particles0 and particles1 (this library's sorted and parts);
- counters, field, blocks.

The CG vectors (fluidCg) are not one: the liquid's pass writes them before
it reads them (js/passes.js:83).

They are laid out as here, so they load as they are. Loading follows
restoreSnapshot (js/snapshot.js:510-548) for these parts:

- a snapshot of another world size is refused;
- one whose particles or counters are laid out otherwise (another
  LIQUID_PER_CELL, an older layout) loads with no particles, its liquid
  cells undrawn so that the next step seeds them afresh (migrateLiquid,
  js/snapshot.js:335-373);
- blocks from before the V-cycle's counts, and a field from before
  viscosity's last sweep, are widened with zeros (migrateBlocks, :391-409;
  migrateField, :448-470);
- any other liquid part of another size is refused, with nothing changed.

A snapshot's other parts (air, heat, bodies, ...) are outside the liquid
step: they are kept, untouched, and written back.
"""
import gzip
import json
import struct

import numpy as np

from . import abi
from . import world as W

MAGIC = b"SANDSNAP"
FORMAT = 1

# this library's buffer name -> the reference's part name (cells: cells{cur})
PART_OF = {"sorted": "particles0", "parts": "particles1", "counters": "counters", "field": "field",
           "blocks": "blocks"}
# the parts dropped, to load empty, when the particles are laid out otherwise
# (js/snapshot.js:61)
LIQUID_PARTS = ("particles0", "particles1", "counters", "blocks")
# the cell word's flags (js/shared.js:79-91)
FLAG_SHIFT, FL_DRAWN = 28, 4


def _align4(n):
    return (n + 3) & ~3


def read(data):
    """A snapshot's (header, parts): parts maps each part's name to its
    bytes (a numpy uint8 array). Raises ValueError on anything this format
    can't read (js/snapshot.js:163-189)."""
    try:
        raw = gzip.decompress(bytes(data))
    except (OSError, EOFError) as e:
        raise ValueError("not a snapshot") from e
    if len(raw) < len(MAGIC) + 4 or raw[:len(MAGIC)] != MAGIC:
        raise ValueError("not a snapshot")
    (length,) = struct.unpack_from("<I", raw, len(MAGIC))
    if len(MAGIC) + 4 + length > len(raw):
        raise ValueError("the snapshot is cut short")
    try:
        header = json.loads(raw[len(MAGIC) + 4:len(MAGIC) + 4 + length].decode())
    except (UnicodeDecodeError, json.JSONDecodeError) as e:
        raise ValueError("not a snapshot") from e
    if not isinstance(header, dict):
        raise ValueError("not a snapshot")
    if header.get("format") != FORMAT:
        raise ValueError(f"saved in snapshot format {header.get('format')}; this reads format {FORMAT}")
    listed = header.get("parts", [])
    if not isinstance(listed, list) or not all(
            isinstance(p, dict) and isinstance(p.get("name"), str) and isinstance(p.get("bytes"), int)
            and not isinstance(p.get("bytes"), bool) and p["bytes"] >= 0 for p in listed):
        raise ValueError("the snapshot's list of parts is malformed")
    parts = {}
    at = len(MAGIC) + 4 + _align4(length)
    for part in listed:
        n = part["bytes"]
        if at + n > len(raw):
            raise ValueError("the snapshot is cut short")
        parts[part["name"]] = np.frombuffer(raw, dtype=np.uint8, count=n, offset=at).copy()
        at += _align4(n)
    return header, parts


def write(header, parts):
    """The gzipped snapshot of `header` (its `parts` list rewritten from
    `parts`, in that dict's order) and `parts` (name -> bytes)."""
    h = dict(header)
    h["format"] = FORMAT
    h["parts"] = [{"name": k, "bytes": int(np.asarray(v).nbytes)} for k, v in parts.items()]
    head = json.dumps(h).encode()
    out = bytearray(MAGIC)
    out += struct.pack("<I", len(head))
    out += head + b"\0" * (_align4(len(head)) - len(head))
    for v in parts.values():
        b = np.ascontiguousarray(v).view(np.uint8).tobytes()
        out += b + b"\0" * (_align4(len(b)) - len(b))
    return gzip.compress(bytes(out))


def _liquid_types(elems):
    """Per cell type id (8 bits), whether the element is a liquid."""
    out = np.zeros(256, dtype=bool)
    for i, e in enumerate(elems):
        out[i] = e.kind == abi.KIND_LIQUID
    return out


def migrate_liquid(world, parts, elems):
    """The parts with the liquid's left out, and its liquid cells undrawn
    with their run word cleared, when particles0 or counters is laid out
    otherwise than world's (js/snapshot.js:335-373). Returns (parts,
    migrated)."""
    saved, counters = parts.get("particles0"), parts.get("counters")
    if saved is None or (saved.nbytes == world.sorted.nbytes and counters is not None
                         and counters.nbytes == world.counters.nbytes):
        return parts, False
    out = {k: v for k, v in parts.items() if k not in LIQUID_PARTS}
    liquid = _liquid_types(elems)
    for name in ("cells0", "cells1"):
        b = parts.get(name)
        if b is None or b.nbytes < 16 * world.C or b.nbytes % 4:
            continue
        u = b.view(np.uint32).copy()
        cell = u[: 4 * world.C].reshape(world.C, 4)
        m = liquid[cell[:, 0] & 0xFF]
        cell[m, 0] &= np.uint32(~(FL_DRAWN << FLAG_SHIFT) & 0xFFFFFFFF)
        cell[m, 3] = 0
        out[name] = u.view(np.uint8)
    return out, True


def migrate_blocks(world, parts):
    """blocks saved with 4 count words after the block lists, not
    FLUID_STATS: the V-cycle's words put in after them, zero
    (js/snapshot.js:391-409)."""
    saved = parts.get("blocks")
    added = (abi.FLUID_STATS - 4) * 4
    if saved is None or saved.nbytes != world.blocks.nbytes - added:
        return parts
    at = (4 * world.L["block_count"] + 4) * 4
    grown = np.zeros(world.blocks.nbytes, dtype=np.uint8)
    grown[:at] = saved[:at]
    grown[at + added:] = saved[at:]
    return dict(parts, blocks=grown)


def migrate_field(world, parts):
    """field saved without viscosity's last sweep per face (a quarter word a
    face after the velocities before viscosity): put in, zero
    (js/snapshot.js:448-470)."""
    saved = parts.get("field")
    F = world.L["face_count"]
    quarter = (F + 3) // 4 * 16
    if saved is None or saved.nbytes != world.field.nbytes - quarter:
        return parts
    at = world.C * 32 + F * 16 + quarter
    grown = np.zeros(world.field.nbytes, dtype=np.uint8)
    grown[:at] = saved[:at]
    grown[at + quarter:] = saved[at:]
    return dict(parts, field=grown)


def _size(header):
    """The header's world size (width, height); ValueError when it has none."""
    try:
        width, height = int(header["width"]), int(header["height"])
    except (KeyError, TypeError, ValueError) as e:
        raise ValueError("the snapshot's header gives no world size") from e
    if width <= 0 or height <= 0:
        raise ValueError(f"the snapshot's world is {width}x{height}")
    return width, height


def restore(world, header, parts, elems=None, element_ids=None):
    """Load a snapshot (read's header and parts) into `world`, a World of its
    size, as restoreSnapshot does for the liquid's parts
    (js/snapshot.js:510-548). `elems` is the element table the cells' type
    ids index (this library's by default); element_ids, when given, the
    host's element ids in that order, which the snapshot's must equal
    (js/snapshot.js:179-181). Raises ValueError, with world unchanged, when
    the elements or the size differ or a liquid part doesn't fit. The
    snapshot's state (frame, tiling parity, iteration count, ...) is kept as
    world.snapshot_state, the rest of its header as world.snapshot_header
    and its other parts as world.snapshot_rest."""
    if element_ids is not None and list(header.get("elements", [])) != list(element_ids):
        raise ValueError("saved with a different set of elements")
    width, height = _size(header)
    if (width, height) != (world.W, world.H):
        raise ValueError(f"the snapshot is of a {width}x{height} world, this one is {world.W}x{world.H}")
    state = header.get("state", {})
    if not isinstance(state, dict) or state.get("cur", 0) not in (0, 1):
        raise ValueError("the snapshot's state names no current cell buffer")
    cur = int(state.get("cur", 0))
    elems = W.element_table() if elems is None else elems
    parts, migrated = migrate_liquid(world, parts, elems)
    parts = migrate_field(world, migrate_blocks(world, parts))
    names = dict(PART_OF, cells=f"cells{cur}")
    misfits = []
    for buf, part in names.items():
        src = parts.get(part)
        if src is None and migrated and part in LIQUID_PARTS:
            continue
        if src is None or src.nbytes != getattr(world, buf).nbytes:
            misfits.append(part)
    other = parts.get(f"cells{1 - cur}")
    if other is not None and other.nbytes != world.cells.nbytes:
        misfits.append(f"cells{1 - cur}")
    if misfits:
        raise ValueError(f"saved by a version that lays out {', '.join(misfits)} differently")
    for buf, part in names.items():
        dst = getattr(world, buf)
        src = parts.get(part)
        if src is None:
            dst[:] = 0
        else:
            dst[:] = src.view(dst.dtype)
    world.cg[:] = 0
    world.snapshot_state = dict(state)
    world.snapshot_elements = list(header.get("elements", []))
    world.snapshot_header = {k: v for k, v in header.items() if k not in ("parts", "state")}
    kept = set(names.values()) | {"cells0", "cells1"} | set(LIQUID_PARTS)
    world.snapshot_rest = {k: v for k, v in parts.items() if k not in kept}
    world.snapshot_other_cells = parts.get(f"cells{1 - cur}")
    world.snapshot_migrated = migrated
    return world


def world_from(header, parts, liquid_per_cell=4, capacity=0, elems=None, element_ids=None):
    """A World of the snapshot's size, with the reference's particle
    capacity for it (or `capacity`), holding the snapshot's liquid
    (restore)."""
    w = W.World(*_size(header), liquid_per_cell, capacity)
    w.config = dict(workload="snapshot", grid=f"{w.W}x{w.H}", seed=0, earth_g=W.earth_g_cells())
    return restore(w, header, parts, elems, element_ids)


def load(data, liquid_per_cell=4, capacity=0, elems=None, element_ids=None):
    """world_from(read(data))."""
    header, parts = read(data)
    return world_from(header, parts, liquid_per_cell, capacity, elems, element_ids)


def save(world, state=None, elements=None):
    """A snapshot of `world`'s liquid (and the other parts and header keys
    it was loaded with, unchanged): its cells as cells0 with `cur` 0 (the
    other cell buffer as loaded, or a copy), the state as given (or as
    loaded, cur set to 0), the elements as loaded (or ids 0..n-1 of this
    library's table)."""
    st = dict(getattr(world, "snapshot_state", {}) if state is None else state)
    st["cur"] = 0
    other = getattr(world, "snapshot_other_cells", None)
    parts = {"cells0": world.cells, "cells1": world.cells.copy() if other is None else other}
    for buf, part in PART_OF.items():
        parts[part] = getattr(world, buf)
    parts.update(getattr(world, "snapshot_rest", {}))
    els = elements if elements is not None else getattr(world, "snapshot_elements", None)
    if els is None:
        els = list(range(len(W.element_table())))
    header = dict(getattr(world, "snapshot_header", {}))
    header.update(format=FORMAT, width=world.W, height=world.H, elements=els, state=st)
    return write(header, parts)


def step_flags(world):
    """The step flags of a loaded world's first step: its tiling parity
    carried on from the saved Simulation.shiftedFirst, which each step flips
    before it relaxes (js/sim.js:2530-2531), set on the handle; later steps
    flip it on the handle as the reference does."""
    st = getattr(world, "snapshot_state", {})
    if "shiftedFirst" not in st:
        return 0
    return abi.STEP_SHIFTED_SET | (abi.STEP_SHIFTED_FIRST if not st["shiftedFirst"] else 0)
