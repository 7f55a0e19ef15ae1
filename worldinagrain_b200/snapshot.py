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
(Simulation.snapshotParts, js/sim.js:1429-1438), a pair named name0 and
name1. The liquid's are:

- cells0 and cells1, the state's `cur` the one the next step reads;
- particles0 and particles1 (this library's sorted and parts);
- counters, field, blocks;
- fluidCg, when the snapshot keeps it.

They are laid out as here, so they load as they are. As in the reference, a
part of another size than this layout gives is refused, not misread
(js/snapshot.js:9-12). A snapshot's other parts (air, heat, bodies, ...)
are outside the liquid step: they are kept, untouched, and written back.
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
           "blocks": "blocks", "cg": "fluidCg"}


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
    try:
        header = json.loads(raw[len(MAGIC) + 4:len(MAGIC) + 4 + length].decode())
    except (UnicodeDecodeError, json.JSONDecodeError) as e:
        raise ValueError("not a snapshot") from e
    if header.get("format") != FORMAT:
        raise ValueError(f"saved in snapshot format {header.get('format')}; this reads format {FORMAT}")
    parts = {}
    at = len(MAGIC) + 4 + _align4(length)
    for part in header.get("parts", []):
        n = int(part["bytes"])
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


def world_from(header, parts, liquid_per_cell=4):
    """A World holding a snapshot's liquid: its size from the header, its
    particle capacity from the particle parts, each buffer the part's bytes.
    The snapshot's state (frame, tiling parity, iteration count, ...) is
    kept as world.snapshot_state and its other parts as world.snapshot_rest.
    Raises ValueError when a liquid part's size differs from this layout's."""
    width, height = int(header["width"]), int(header["height"])
    state = header.get("state", {})
    cur = int(state.get("cur", 0))
    p0 = parts.get("particles0")
    if p0 is None or p0.nbytes < 16 or (p0.nbytes - 16) % 48:
        raise ValueError("the snapshot has no particle buffer of this layout")
    cap = (p0.nbytes - 16) // 48
    w = W.World(width, height, liquid_per_cell, cap)
    names = dict(PART_OF, cells=f"cells{cur}")
    for buf, part in names.items():
        dst = getattr(w, buf)
        src = parts.get(part)
        if src is None:
            if buf == "cg":  # not kept: cgStart writes it before any pass reads it
                continue
            raise ValueError(f"the snapshot has no {part}")
        if src.nbytes != dst.nbytes:
            raise ValueError(f"{part} is {src.nbytes} bytes; this layout's {buf} is {dst.nbytes}")
        dst[:] = src.view(dst.dtype)
    w.config = dict(workload="snapshot", grid=f"{width}x{height}", seed=0, earth_g=W.earth_g_cells())
    w.snapshot_state = dict(state)
    w.snapshot_elements = list(header.get("elements", []))
    w.snapshot_rest = {k: v for k, v in parts.items()
                       if k not in set(names.values()) and not (k.startswith("cells") and k[5:] in ("0", "1"))}
    w.snapshot_other_cells = parts.get(f"cells{1 - cur}")
    return w


def load(data, liquid_per_cell=4):
    """world_from(read(data))."""
    header, parts = read(data)
    return world_from(header, parts, liquid_per_cell)


def save(world, state=None, elements=None):
    """A snapshot of `world`'s liquid (and the other parts it was loaded
    with, unchanged): its cells as cells0 with `cur` 0 (the other cell
    buffer as loaded, or a copy), the state as given (or as loaded, cur set
    to 0), the elements as loaded (or ids 0..n-1 of this library's table)."""
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
    header = {"format": FORMAT, "width": world.W, "height": world.H, "elements": els, "state": st}
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
