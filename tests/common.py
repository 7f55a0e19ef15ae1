"""Shared helpers of the tests: worlds, and comparisons of two worlds'
buffers (grid words bit for bit; particles as multisets, the within-cell
order and the sort slot being an atomic's order in the reference too,
shaders/fluid.wgsl:3707)."""
import numpy as np

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

GRID = ("cells", "counters", "field", "blocks", "cg")


def canonical_particles(world, which):
    """Live particles of a Particles buffer as a sorted array of rows
    (motion bits, state bits with the sort slot masked, affine bits)."""
    buf = getattr(world, which)
    n = min(int(buf[0]), world.cap)
    items = buf[4:].reshape(3, world.cap, 4)
    rows = np.concatenate([items[0, :n], items[1, :n], items[2, :n]], axis=1).astype(np.uint64)
    rows[:, 7] = 0  # state.w: the slot sortCount's atomic gave it
    if n == 0:
        return rows
    order = np.lexsort(rows.T[::-1])
    return rows[order]


def run_membership(world):
    """For `sorted`: whether every live particle sits in its cell's run
    (G_START .. G_START + G_SORT)."""
    n = min(int(world.sorted[0]), world.cap)
    if n == 0:
        return True
    m = world.sorted[4:].reshape(3, world.cap, 4)[0, :n].view(np.float32)
    cx = np.clip(np.floor(m[:, 0]).astype(np.int64), 0, world.W - 1)
    cy = np.clip(np.floor(m[:, 1]).astype(np.int64), 0, world.H - 1)
    cell = cy * world.W + cx
    cc = world.counters_cells()
    start = cc[cell, 3].astype(np.int64)
    count = cc[cell, 2].astype(np.int64)
    k = np.arange(n)
    return bool(np.all((k >= start) & (k < start + count)))


def diff_words(a, b, name, limit=8):
    a = np.ascontiguousarray(a).view(np.uint32)
    b = np.ascontiguousarray(b).view(np.uint32)
    if a.shape != b.shape:
        return f"{name}: shapes {a.shape} vs {b.shape}"
    bad = np.nonzero(a != b)[0]
    if bad.size == 0:
        return None
    fa, fb = a.view(np.float32), b.view(np.float32)
    head = ", ".join(f"[{i}] {a[i]:#x}({fa[i]:.7g}) vs {b[i]:#x}({fb[i]:.7g})" for i in bad[:limit])
    return f"{name}: {bad.size} words differ: {head}"


def canonical_regions(counters, C):
    """counters with each cell's G_REGION link (word 1) replaced by its
    union-find root (label.wgsl: a link is to a lower index; a word not below
    its index is a root).  Which intermediate links a lock-free union-find
    leaves hangs on thread timing; the roots, which are all the passes read
    (ufFind), do not."""
    out = np.array(counters, copy=True)
    words = out[: 11 * C].reshape(C, 11)[:, 1].astype(np.int64)
    idx = np.arange(C, dtype=np.int64)
    parent = np.where(words < idx, words, idx)
    for _ in range(64):
        nxt = parent[parent]
        if np.array_equal(nxt, parent):
            break
        parent = nxt
    canon = np.where(parent != idx, parent, words).astype(np.uint32)
    out[: 11 * C].reshape(C, 11)[:, 1] = canon
    return out


def mask_solve_scratch(world, name, arr):
    """arr with the pressure solve's scratch words zeroed: what a step writes
    for its own later passes and the next step overwrites before it reads
    them — the relaxation's rim snapshot (counters' G_RIM, words 9-10 of a
    cell), the coarse levels (field past the faces), and cg's per-block
    partial sums and scalars.  The fast form keeps these in its own scratch."""
    a = np.array(arr, copy=True)
    C, L = world.C, world.L
    if name == "counters":
        a[: 11 * C].reshape(C, 11)[:, 9:11] = 0
    elif name == "field":
        F = L["face_count"]
        start = 4 * (2 * C + F + 2 * ((F + 3) // 4))
        a[start:] = 0
    elif name == "cg":
        a[4 * C:] = 0
    return a


def compare_worlds(x, y, grid=GRID, particles=("sorted", "parts"), skip_parts=False, region_links=False,
                   scratch=False):
    """A list of differences between worlds x and y (empty when equal).
    region_links: compare the G_REGION words by their roots; scratch: leave
    out the solve's scratch words (mask_solve_scratch)."""
    out = []
    for name in grid:
        a, b = getattr(x, name), getattr(y, name)
        if scratch:
            a, b = mask_solve_scratch(x, name, a), mask_solve_scratch(y, name, b)
        if region_links and name == "counters":
            a, b = canonical_regions(a, x.C), canonical_regions(b, y.C)
        d = diff_words(a, b, name)
        if d:
            out.append(d)
    for which in particles:
        if skip_parts and which == "parts":
            continue
        if int(getattr(x, which)[0]) != int(getattr(y, which)[0]):
            out.append(f"{which}.count {int(getattr(x, which)[0])} vs {int(getattr(y, which)[0])}")
            continue
        px, py = canonical_particles(x, which), canonical_particles(y, which)
        if px.shape != py.shape or not np.array_equal(px, py):
            nbad = int(np.sum(np.any(px != py, axis=1))) if px.shape == py.shape else -1
            out.append(f"{which}: particle multisets differ ({nbad} rows)")
    return out


def params(world, step, seed=0x1234):
    return W.make_params(world, frame=step, seed=seed, earth_g=world.config["earth_g"])


def busy_world(width=48, height=40, seed=11):
    """A small world with walls, obstacles and moving water, for parity."""
    return W.small_world(width, height, seed=seed, kind="obstacles")
