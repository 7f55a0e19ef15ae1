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

The free bodies' parts (bodyMotion, the body table; bodies, the bodies'
buffer with its swept stamps) are migrated as restoreSnapshot migrates
them (migrateSwept, migrateTable, migrateBodies, js/snapshot.js:411-507:
the last one lets go the loose cells of a snapshot from before its bodies
were kept whole, which the liquid step reads), kept, and handed to a host
that binds them (bodies_from); keep_bodies puts the stepped table back for
`save`. A snapshot's other parts (air, heat, ...) are outside the liquid
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


# The bodies' parts (js/snapshot.js:411-507): header.bodies, whether the
# snapshot's bodies were kept whole; the width of a body's slot before the
# contacts' mobility was added; a loose cell's slot once its body let it go.
BODIES = 1
OLD_TABLE_WORDS = 108
FREE_BODY = 2047.0


def _body_sizes(world):
    """(bytes of bodyMotion, of the bodies buffer, of a cell's two swept
    words over the world, of the table's growth past OLD_TABLE_WORDS)."""
    stamps_words, _ = abi.body_stamps_layout(world.W, world.H)
    return (4 * abi.BODY_MOTION_WORDS, 4 * stamps_words, 2 * 4 * world.C,
            4 * abi.MAX_BODIES * (abi.BODY_TABLE_WORDS - OLD_TABLE_WORDS))


def migrate_swept(world, parts):
    """A snapshot from before the swept stamps moved to the end of the
    bodies buffer (two words a cell at the start of bodyMotion then): those
    dropped from bodyMotion, and none at the end of bodies, so no cell is
    taken as a cup of last step's (migrateSwept, js/snapshot.js:411-426)."""
    motion_bytes, bodies_bytes, cell_bytes, growth = _body_sizes(world)
    bodies, motion = parts.get("bodies"), parts.get("bodyMotion")
    if (bodies is None or motion is None or bodies.nbytes != bodies_bytes - cell_bytes
            or motion.nbytes not in (motion_bytes + cell_bytes, motion_bytes - growth + cell_bytes)):
        return parts
    grown = np.zeros(bodies_bytes, dtype=np.uint8)
    grown[:bodies.nbytes] = bodies
    return dict(parts, bodies=grown, bodyMotion=motion[cell_bytes:].copy())


def migrate_table(world, parts):
    """A snapshot whose body slots were OLD_TABLE_WORDS wide: each slot
    widened with zeros (no contact mobility worked out: a body gives way by
    its mass alone until the bodies' pass has run), the contacts and the
    liquid's words after the table moved along (migrateTable,
    js/snapshot.js:428-450)."""
    motion_bytes, _, _, growth = _body_sizes(world)
    saved = parts.get("bodyMotion")
    if saved is None or saved.nbytes != motion_bytes - growth:
        return parts
    nb, old_w, new_w = abi.MAX_BODIES, OLD_TABLE_WORDS, abi.BODY_TABLE_WORDS
    old = saved.view(np.uint32)
    grown = np.zeros(abi.BODY_MOTION_WORDS, dtype=np.uint32)
    grown[:nb] = old[:nb]
    grown[nb:nb * (1 + new_w)].reshape(nb, new_w)[:, :old_w] = old[nb:nb * (1 + old_w)].reshape(nb, old_w)
    grown[nb * (1 + new_w):] = old[nb * (1 + old_w):]
    return dict(parts, bodyMotion=grown.view(np.uint8))


def migrate_bodies(world, header, parts, cur, elems):
    """A snapshot from before its bodies were kept whole (header.bodies under
    BODIES): every live body looked at whole in its first step (BF_PARTS),
    and each loose solid cell its body did not stamp in its last step (its
    claim word is not the body's key) let go as a broken body's are, its
    slot FREE_BODY (migrateBodies, js/snapshot.js:471-507).  The liquid step
    reads the slot: a cell let go is no body's."""
    motion_bytes, bodies_bytes, _, _ = _body_sizes(world)
    name = f"cells{cur}"
    saved, bodies, motion = parts.get(name), parts.get("bodies"), parts.get("bodyMotion")
    if (int(header.get("bodies", 0)) >= BODIES or saved is None or bodies is None or motion is None
            or bodies.nbytes != bodies_bytes or motion.nbytes != motion_bytes or saved.nbytes < 16 * world.C):
        return parts
    nb, tw = abi.MAX_BODIES, abi.BODY_TABLE_WORDS
    table = motion.view(np.uint32).copy()
    flags = table[nb:nb * (1 + tw)].reshape(nb, tw)[:, abi.BW["FLAGS"]]
    alive = (flags & abi.BF_ALIVE) != 0
    flags[alive] |= 8  # BODY_FLAG.PARTS (js/shared.js:327)
    table[nb:nb * (1 + tw)].reshape(nb, tw)[:, abi.BW["FLAGS"]] = flags
    tiles = -(-world.W // abi.BODY_TILE) * -(-world.H // abi.BODY_TILE)
    body_header = 4 * tiles + abi.BODY_STAT_WORDS + abi.BODY_COUNTERS + nb
    claims = bodies.view(np.uint32)[body_header + world.C:body_header + 2 * world.C]
    cells = saved.view(np.uint32).copy()
    cell = cells[:4 * world.C].reshape(world.C, 4)
    kind = np.array([elems[t].kind if t < len(elems) else elems[0].kind for t in range(256)])
    slot = (cell[:, 3] & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float64)
    loose = (((cell[:, 0] >> FLAG_SHIFT) & abi.FL_LOOSE) != 0) & (kind[cell[:, 0] & 0xFF] == abi.KIND_SOLID) & (slot < nb)
    for i in np.flatnonzero(loose):
        # (a slot that is no whole number of the table, which only a damaged
        # snapshot holds, is let go: its body words are none)
        b = int(slot[i])
        whole = slot[i] >= 0 and slot[i] == b
        body = table[nb + b * tw:nb + (b + 1) * tw] if whole else np.zeros(tw, dtype=np.uint32)
        key = (((int(body[abi.BW["FRAME"]]) & 0xFFFFF) << 12) | (int(FREE_BODY - slot[i]) << 1)) & 0xFFFFFFFF
        if not (body[abi.BW["FLAGS"]] & abi.BF_ALIVE) or int(claims[i]) != key:
            cell[i, 3] = (int(cell[i, 3]) & 0xFFFF0000) | int(np.float16(FREE_BODY).view(np.uint16))
    return dict(parts, **{name: cells.view(np.uint8), "bodyMotion": table.view(np.uint8)})


def bodies_from(world):
    """The free bodies of a world restored from a snapshot, as a world.Bodies
    to bind (LiquidStep.bind_bodies): its body table and bodies' buffer as
    saved (after the migrations above), the push sums empty (a step's
    scratch, not a part).  None when the snapshot holds no body parts of
    this world's layout."""
    rest = getattr(world, "snapshot_rest", {})
    motion_bytes, bodies_bytes, _, _ = _body_sizes(world)
    motion, stamps = rest.get("bodyMotion"), rest.get("bodies")
    if motion is None or stamps is None or motion.nbytes != motion_bytes or stamps.nbytes != bodies_bytes:
        return None
    b = W.Bodies(world.W, world.H)
    b.motion[:] = motion.view(np.uint32)
    b.stamps[:] = stamps.view(np.uint32)
    return b


def keep_bodies(world, bodies):
    """The stepped body table (what the liquid did to each body in its
    liquid words) into the parts `save` writes back."""
    world.snapshot_rest = dict(getattr(world, "snapshot_rest", {}), bodyMotion=bodies.motion.view(np.uint8).copy())


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
    parts = migrate_table(world, migrate_swept(world, migrate_blocks(world, parts)))
    parts = migrate_bodies(world, header, migrate_field(world, parts), cur, elems)
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
    header.update(format=FORMAT, width=world.W, height=world.H, elements=els, state=st, bodies=BODIES)
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
