"""Host-side world state in the reference's buffer layouts, and the
synthetic worlds of the benchmark configurations.

A world is the set of buffers `Simulation` allocates for the liquid
(js/sim.js:741-843) plus the `cells` raster, all as numpy arrays in the exact
byte layouts the shaders read:

  cells     u32[4 * (C + ceil(C/2))]   vec4 per cell (x word, temp bits, f16x2
                                       velocity, w), then the gas plane
  sorted    u32[4 + 12 * cap]          Particles: count, 3 pad, motion/state/affine planes
  parts     u32[4 + 12 * cap]
  counters  u32[11 C + 2 F]
  field     f32[4 * (2 (C + level cells) + F + 2 ceil(F/4))]
  blocks    u32[5 B + 9]
  cg        f32[4 * (C + B + 1)]

New liquid is painted as undrawn WATER cells, and the first step's syncSeed
(shaders/fluid.wgsl:863-890) turns each into LIQUID_PER_CELL particles, as a
scene painted by js/scenes.js is (`dam`, js/scenes.js:404-407).
"""
import ctypes as C
import math
import struct

import numpy as np

from . import abi

# ---------------------------------------------------------------- elements

GRAVITY = 9.81 / 3600 / 0.01  # js/elements.js:31, cells/step^2 at 1 cm and 60 steps/s
T_NEVER = 1e9
GAS_HEAT_CAP = 1.2e-3 * 1000.0  # order of js/shared.js:174; read by nothing on the liquid's path


MUD = 4  # a viscous liquid of this table's own (not the reference's id)


def element_table():
    """The element rows the liquid step reads, for AIR, WALL, SAND, WATER
    (js/elements.js:414-458, with DEFAULTS js/elements.js:316-360), and a
    fifth, a viscous liquid denser than water (on the lines of the
    reference's mud, js/elements.js:510-514) for the viscosity passes."""
    rows = [abi.Elem() for _ in range(5)]

    def fill(e, **kw):
        base = dict(kind=abi.KIND_SOLID, density=1000.0, weight=GRAVITY, heat_cap=2.0, viscosity=0.0,
                    viscosity_t=20.0, viscosity_e=0.0, tension=0.0, expansion=0.0, expansion2=0.0,
                    hi_t=T_NEVER, lo_t=-T_NEVER, up_span=1e30, down_span=1e30, down_scale=0.0,
                    sol_density=0.0, flags=0, wetting=0.5, break_to=abi.NO_ELEM)
        base.update(kw)
        for k, v in base.items():
            setattr(e, k, v)

    fill(rows[abi.AIR], kind=abi.KIND_GAS, density=1.0, weight=0.0, heat_cap=GAS_HEAT_CAP)
    fill(rows[abi.WALL], flags=4 | 2 | 8, wetting=0.8)
    fill(rows[abi.SAND], kind=abi.KIND_POWDER, density=265.0, heat_cap=1.3, hi_t=1250.0, wetting=0.95,
         up_span=220.0 / 1.3)
    fill(rows[abi.WATER], kind=abi.KIND_LIQUID, density=100.0, heat_cap=4.18, hi_t=100.0, lo_t=0.0,
         up_span=2257.0 / 4.18, down_span=334.0 / 4.18, down_scale=1.0, expansion=1.42e-4,
         expansion2=4.45e-6, tension=1.0, flags=2)
    fill(rows[MUD], kind=abi.KIND_LIQUID, density=160.0, heat_cap=3.3, viscosity=0.8, hi_t=T_NEVER, lo_t=-T_NEVER)
    return (abi.Elem * 5)(*rows)


# ---------------------------------------------------------------- cells

def f32_bits(x):
    return struct.unpack("<I", struct.pack("<f", float(x)))[0]


def f16x2(a, b):
    """pack2x16float of float arrays a, b (round to nearest even)."""
    lo = np.asarray(a, dtype=np.float32).astype(np.float16).view(np.uint16).astype(np.uint32)
    hi = np.asarray(b, dtype=np.float32).astype(np.float16).view(np.uint16).astype(np.uint32)
    return lo | (hi << 16)


class World:
    """The liquid's buffers for one world, host side, zeroed as
    Simulation.clear leaves them (js/sim.js:1259)."""

    def __init__(self, width, height, liquid_per_cell=4, capacity=0, temperature=20.0):
        self.L = abi.layout_py(width, height, liquid_per_cell, capacity)
        L = self.L
        self.W, self.H = L["width"], L["height"]
        self.C = L["cell_count"]
        self.cap = L["capacity"]
        self.cells = np.zeros(L["cells_bytes"] // 4, dtype=np.uint32)
        self.sorted = np.zeros(L["particles_bytes"] // 4, dtype=np.uint32)
        self.parts = np.zeros(L["particles_bytes"] // 4, dtype=np.uint32)
        self.counters = np.zeros(L["counters_bytes"] // 4, dtype=np.uint32)
        self.field = np.zeros(L["field_bytes"] // 4, dtype=np.float32)
        self.blocks = np.zeros(L["blocks_bytes"] // 4, dtype=np.uint32)
        self.cg = np.zeros(L["cg_bytes"] // 4, dtype=np.float32)
        cv = self.cell_view()
        cv[:, 0] = abi.AIR
        cv[:, 1] = f32_bits(temperature)
        self.temperature = temperature

    def desc(self):
        return abi.WorldDesc(self.W, self.H, self.L["liquid_per_cell"], self.cap)

    def cell_view(self):
        return self.cells[: 4 * self.C].reshape(self.H, self.W, 4)

    def paint(self, mask, elem, vel=None):
        """Cells under mask (H x W bool) become `elem`, undrawn, at the
        world's temperature; vel (H x W x 2, cells/step) sets their f16
        velocity, which syncSeed gives the particles it seeds there."""
        cv = self.cell_view()
        cv[mask, 0] = elem
        cv[mask, 1] = f32_bits(self.temperature)
        cv[mask, 3] = 0
        if vel is not None:
            cv[mask, 2] = f16x2(vel[..., 0][mask], vel[..., 1][mask])
        else:
            cv[mask, 2] = 0

    def buffers(self):
        return {k: getattr(self, k) for k in abi.BUFFER_NAMES}

    def copy(self):
        w = World.__new__(World)
        w.__dict__.update(self.__dict__)
        for k in abi.BUFFER_NAMES:
            setattr(w, k, getattr(self, k).copy())
        return w

    # -- views used by the tests
    def particle_count(self, which="sorted"):
        return int(getattr(self, which)[0])

    def particles(self, which="sorted"):
        """(motion f32[n,4], state u32[n,4], affine f32[n,4]) of the live particles."""
        buf = getattr(self, which)
        n = min(int(buf[0]), self.cap)
        items = buf[4:].reshape(3, self.cap, 4)
        return (items[0, :n].view(np.float32), items[1, :n], items[2, :n].view(np.float32))

    def counters_cells(self):
        return self.counters[: 11 * self.C].reshape(self.C, 11)

    def field_cells(self):
        return self.field[: 8 * self.C].reshape(self.C, 2, 4)

    def pressure(self):
        return self.field_cells()[:, 0, 0].reshape(self.H, self.W)

    def density_class(self):
        return self.field_cells()[:, 0, 2].reshape(self.H, self.W)


def make_params(world, frame, seed, earth_g, dx=1.0, dt=1.0 / 120.0):
    P = abi.Params()
    P.size[0], P.size[1] = world.W, world.H
    P.frame = frame & 0xffffffff
    P.seed = seed & 0xffffffff
    P.dx = dx
    P.earth_g = earth_g
    P.dt = dt
    return P


# ---------------------------------------------------------------- configurations

def earth_g_cells(g=9.8, dt=1.0 / 120.0, dx=1.0):
    """|g| dt^2 / dx: the Earth's pull in cells per step^2 (y down)."""
    return float(np.float32(g * dt * dt / dx))


def dam_break(width=256, height=256, seed=1):
    """Plain 2D dam break: one-cell WALL border, WATER filling the bottom-left
    40% width x 60% height inside it, at rest (4 particles per cell seeded by
    syncSeed's jittered quarters)."""
    w = World(width, height)
    wall = np.zeros((height, width), dtype=bool)
    wall[0, :] = wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    w.paint(wall, abi.WALL)
    fw, fh = int(round(0.4 * width)), int(round(0.6 * height))
    water = np.zeros((height, width), dtype=bool)
    water[height - 1 - fh:height - 1, 1:1 + fw] = True
    w.paint(water, abi.WATER)
    w.config = dict(workload="dam_break", grid=f"{width}x{height}", seed=seed, earth_g=earth_g_cells())
    return w


def disks_world(width=1024, height=1024, n_disks=200, r_lo=4, r_hi=24, sigma=0.5, seed=2):
    """Single world at scale: WALL disks (centres and radii uniform under the
    seed), WATER in the top half outside them with Gaussian cell velocities
    (sigma cells/step per axis, one draw per cell, carried by the cell's f16
    velocity into the 4 particles syncSeed puts there)."""
    rng = np.random.default_rng(seed)
    w = World(width, height)
    yy, xx = np.mgrid[0:height, 0:width]
    wall = np.zeros((height, width), dtype=bool)
    cx = rng.uniform(0, width, n_disks)
    cy = rng.uniform(0, height, n_disks)
    r = rng.uniform(r_lo, r_hi, n_disks)
    for k in range(n_disks):
        x0, x1 = int(max(0, cx[k] - r[k] - 1)), int(min(width, cx[k] + r[k] + 2))
        y0, y1 = int(max(0, cy[k] - r[k] - 1)), int(min(height, cy[k] + r[k] + 2))
        sub = (xx[y0:y1, x0:x1] + 0.5 - cx[k]) ** 2 + (yy[y0:y1, x0:x1] + 0.5 - cy[k]) ** 2 <= r[k] ** 2
        wall[y0:y1, x0:x1] |= sub
    w.paint(wall, abi.WALL)
    water = (yy < height // 2) & ~wall
    vel = rng.normal(0.0, sigma, (height, width, 2)).astype(np.float32)
    w.paint(water, abi.WATER, vel=vel)
    w.config = dict(workload="disks", grid=f"{width}x{height}", seed=seed, earth_g=earth_g_cells(),
                    disks=n_disks, sigma=sigma)
    return w


def obstacle_column(width=2048, height=2048, p_solid=0.03, fill=0.7, ppc=2, seed=3):
    """Mixed-precision config: Bernoulli(p) WALL cells dilated once (4-neighbour),
    WATER in the bottom `fill` of the height outside them, `ppc` particles per
    cell (LIQUID_PER_CELL as a parameter)."""
    rng = np.random.default_rng(seed)
    w = World(width, height, liquid_per_cell=ppc)
    seedm = rng.random((height, width)) < p_solid
    wall = seedm.copy()
    wall[1:, :] |= seedm[:-1, :]
    wall[:-1, :] |= seedm[1:, :]
    wall[:, 1:] |= seedm[:, :-1]
    wall[:, :-1] |= seedm[:, 1:]
    w.paint(wall, abi.WALL)
    yy = np.arange(height)[:, None]
    water = (yy >= height - int(round(fill * height))) & ~wall
    w.paint(water, abi.WATER)
    w.config = dict(workload="obstacle_column", grid=f"{width}x{height}", seed=seed, earth_g=earth_g_cells(),
                    p_solid=p_solid, ppc=ppc)
    return w


def multi_world_specs(n=512, lo=64, hi=512, seed=4, ppc=4):
    """The shapes multi_worlds draws, without building the worlds: per world
    (side, kind, fluid fraction, fluid block width and height, particle
    capacity)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        s = int(16 * round(lo * (hi / lo) ** rng.uniform() / 16))
        kind = "dam" if rng.uniform() < 0.5 else "column"
        f = rng.uniform(0.2, 0.7)
        inner = s - 2
        if kind == "dam":
            fh = min(inner, int(round(inner * min(0.95, (1.5 * f) ** 0.5))))
            fw = min(inner, int(round(f * inner * inner / max(fh, 1))))
        else:
            fw, fh = inner, min(inner, int(round(f * inner)))
        cap = int(np.ceil(fw * fh * ppc * 1.25)) + 256
        out.append((s, kind, float(f), fw, fh, cap))
    return out


def multi_worlds(n=512, lo=64, hi=512, seed=4, ppc=4, only=None):
    """Batched multi-world config: n independent square worlds, sides
    log-uniform in [lo, hi] rounded to a multiple of 16, each a dam break
    (WATER against the left wall, about 1.5 times as high as wide) or a
    column (the bottom rows, full width), fluid fraction U(0.2, 0.7) of the
    inside, at rest, ppc particles per fluid cell, one-cell WALL border.  The
    particle buffers are sized to the liquid (1.25 times its particles), not
    to the whole grid.  `only`: build just these of the n worlds."""
    specs = multi_world_specs(n, lo, hi, seed, ppc)
    out = []
    for k in (range(n) if only is None else only):
        s, kind, f, fw, fh, cap = specs[k]
        w = World(s, s, ppc, cap)
        wall = np.zeros((s, s), dtype=bool)
        wall[0, :] = wall[-1, :] = True
        wall[:, 0] = wall[:, -1] = True
        w.paint(wall, abi.WALL)
        water = np.zeros((s, s), dtype=bool)
        water[s - 1 - fh:s - 1, 1:1 + fw] = True
        w.paint(water, abi.WATER)
        w.config = dict(workload=f"multi_{kind}", grid=f"{s}x{s}", seed=seed, earth_g=earth_g_cells(), fill=f, index=k)
        out.append(w)
    return out


def two_liquids(width=40, height=32, seed=5):
    """Water on the left and a viscous liquid (MUD) on the right of a walled
    box, moving: two liquids in contact, their cells rasterised by the most
    numerous, the viscous one's faces swept (viscosityRed/Black, unpress)."""
    rng = np.random.default_rng(seed)
    w = World(width, height)
    wall = np.zeros((height, width), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    w.paint(wall, abi.WALL)
    vel = rng.normal(0.0, 0.3, (height, width, 2)).astype(np.float32)
    water = np.zeros((height, width), dtype=bool)
    water[height // 3:height - 1, 1:width // 2] = True
    w.paint(water, abi.WATER, vel=vel)
    mud = np.zeros((height, width), dtype=bool)
    mud[height // 2:height - 1, width // 2:width - 1] = True
    w.paint(mud, MUD, vel=vel)
    w.config = dict(workload="two_liquids", grid=f"{width}x{height}", seed=seed, earth_g=earth_g_cells())
    return w


def small_world(width=32, height=32, seed=7, kind="dam"):
    """A small world for parity tests: walls, a block of water and a few
    obstacles, sized so the oracle finishes in well under a second a step."""
    rng = np.random.default_rng(seed)
    w = World(width, height)
    wall = np.zeros((height, width), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    if kind == "obstacles":
        for _ in range(max(1, width * height // 300)):
            x, y = rng.integers(2, width - 3), rng.integers(height // 2, height - 3)
            wall[y:y + 2, x:x + 2] = True
    w.paint(wall, abi.WALL)
    water = np.zeros((height, width), dtype=bool)
    water[height // 3:height - 1, 1:width // 2] = True
    water &= ~wall
    vel = None
    if kind in ("obstacles", "moving"):
        vel = rng.normal(0.0, 0.5, (height, width, 2)).astype(np.float32)
    w.paint(water, abi.WATER, vel=vel)
    w.config = dict(workload=f"small_{kind}", grid=f"{width}x{height}", seed=seed, earth_g=earth_g_cells())
    return w


# ---------------------------------------------------------------- free bodies

WOOD = 5  # a structural solid of this table's own that the test bodies are made of


def body_element_table():
    """element_table() and a sixth row: a structural solid lighter than water
    on the lines of the reference's wood (density 60, breakTo an element,
    js/elements.js:608-614).  A breakTo is what lets a loose cell of it be a
    free body's (fluid.wgsl:1233-1248); SAND stands in for the sawdust this
    table does not have."""
    base = element_table()
    rows = (abi.Elem * 6)()
    for k in range(5):
        C.memmove(C.byref(rows[k]), C.byref(base[k]), C.sizeof(abi.Elem))
    C.memmove(C.byref(rows[WOOD]), C.byref(base[abi.WALL]), C.sizeof(abi.Elem))
    rows[WOOD].density = 60.0
    rows[WOOD].break_to = abi.SAND
    return rows


class Bodies:
    """A free-body table (binding 12, `motion`), the solve's push sums
    (binding 16, `pushes`) and the bodies' buffer of a world (binding 14,
    `stamps`, of which the liquid step reads the swept stamps) in the
    reference's layouts (js/shared.js:294-333, js/sim.js:796-799), host
    side.  The liquid step reads a body's pose, motion, mass and flags and
    adds what it does to the body into the body's liquid words."""

    def __init__(self, width, height):
        self.motion = np.zeros(abi.BODY_MOTION_WORDS, dtype=np.uint32)
        self.pushes = np.zeros(abi.MAX_BODIES * abi.BODY_PUSH_WORDS, dtype=np.uint32)
        words, self.stamp_at = abi.body_stamps_layout(width, height)
        self.stamps = np.zeros(words, dtype=np.uint32)
        self.width = width
        self.swept = []  # (cells' flat indices, body, seam) stamped every step (stamp_step)

    def stamp(self, frame, cells, b, seam):
        """Cells (flat indices) swept by body b at step `frame`, as its cup or
        as seams of its wall (bodies.wgsl's stamp: claimStep(frame) << 12 |
        (2047 - b) << 1 | seam)."""
        key = ((frame % abi.CLAIM_PERIOD + 1) << 12) | ((2047 - b) << 1) | (1 if seam else 0)
        self.stamps[self.stamp_at + 2 * np.asarray(cells, dtype=np.int64) + (frame & 1)] = key

    def stamp_step(self, frame):
        """The stamps the bodies would leave at step `frame` (the bodies
        here stand still, so the same cells each step)."""
        for cells, b, seam in self.swept:
            self.stamp(frame, cells, b, seam)

    def words(self, b):
        at = abi.MAX_BODIES + b * abi.BODY_TABLE_WORDS
        return self.motion[at:at + abi.BODY_TABLE_WORDS]

    def liquid(self, b):
        """The body's liquid words: its change in velocity x, y and spin in
        RIGID_FIX fixed point (i32), and the wet word."""
        at = abi.BODY_LIQUID_BASE + b * abi.BODY_LIQUID_WORDS
        return self.motion[at:at + abi.BODY_LIQUID_WORDS]

    def set_f32(self, b, k, *values):
        self.words(b)[k:k + len(values)] = np.asarray(values, dtype=np.float32).view(np.uint32)

    def copy(self):
        o = Bodies.__new__(Bodies)
        o.__dict__.update(self.__dict__)
        o.motion = self.motion.copy()
        o.pushes = self.pushes.copy()
        o.stamps = self.stamps.copy()
        return o


def stamp_body(world, bodies, b, mask, density, vel=(0.0, 0.0), spin=0.0, subcell=(0.0, 0.0), flags=abi.BF_ALIVE,
               mobility=None, mobility_at=0xffffffff):
    """Body b's cells (mask, H x W) stamped as loose WOOD cells carrying its
    slot in frac.x (shaders/common.wgsl:113-160), and its table slot: pose
    at the cells' centre of mass, velocity and spin, mass (density in water
    cells a cell) and moment of inertia about the centre, flags, the pose's
    sub-cell offset, and optionally a contact mobility (6 f32 of a symmetric
    3 x 3) worked out at step mobility_at."""
    ys, xs = np.nonzero(mask)
    cx, cy = xs + 0.5, ys + 0.5
    n = len(xs)
    m = np.float32(density) * np.float32(n)
    pos = (np.float32(cx.mean()), np.float32(cy.mean()))
    inertia = np.float32(density * np.sum((cx - pos[0]) ** 2 + (cy - pos[1]) ** 2 + 1.0 / 6.0))
    cv = world.cell_view()
    cv[mask, 0] = WOOD | (abi.FL_LOOSE << 28)
    cv[mask, 1] = f32_bits(world.temperature)
    cv[mask, 2] = 0
    cv[mask, 3] = f16x2(np.full(n, float(b)), np.zeros(n))
    bodies.set_f32(b, abi.BW["POS"], *pos)
    bodies.set_f32(b, abi.BW["VEL"], *vel)
    bodies.set_f32(b, abi.BW["SPIN"], spin)
    bodies.set_f32(b, abi.BW["MASS"], m)
    bodies.set_f32(b, abi.BW["INERTIA"], inertia)
    bodies.words(b)[abi.BW["CELLS"]] = n
    bodies.words(b)[abi.BW["FLAGS"]] = flags
    bodies.words(b)[abi.BW["SUBCELL"]] = f16x2(np.array([subcell[0]]), np.array([subcell[1]]))[0]
    if mobility is not None:
        bodies.set_f32(b, abi.BW["MOBILITY"], *mobility)
    bodies.words(b)[abi.BW["MOBILITY_AT"]] = mobility_at & 0xffffffff


def bodies_world(width=96, height=80, seed=6, liquid=abi.WATER, stamps=True):
    """A tank of water with synthetic free bodies in it (none of the
    reference's configs has any): a plank afloat at the surface, moving and
    spinning, with a sub-cell pose; a block under the water whose contact
    mobility was worked out the step before the first, with a seam its stamp
    opened in its wall; a heavy block held on the floor, wet; a body just
    found (NEW, a wall until weighed); cells of a slot that is not alive;
    and a hull afloat whose cup holds sand (its cargo) and the water over
    its rim.  liquid: the tank's liquid (MUD for the viscous sweeps and the
    liquid's drag on the bodies).  stamps: the hull's cup and the block's
    seam in the swept stamps (Bodies.stamp_step writes them a step).
    Returns (world, bodies)."""
    rng = np.random.default_rng(seed)
    w = World(width, height)
    bodies = Bodies(width, height)
    wall = np.zeros((height, width), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    w.paint(wall, abi.WALL)
    surface = height // 3
    used = wall.copy()

    def box(x0, y0, bw, bh):
        m = np.zeros((height, width), dtype=bool)
        m[y0:y0 + bh, x0:x0 + bw] = True
        assert not np.any(m & used)
        used[m] = True
        return m

    stamp_body(w, bodies, 0, box(width // 6, surface - 1, 14, 3), 0.6, vel=(0.05, 0.03), spin=0.002,
               subcell=(0.25, -0.125))
    block = box(width // 2, surface + 12, 6, 6)
    seam = np.zeros_like(block)
    seam[surface + 14, width // 2 + 2] = True  # a gap in the block's wall, left to the liquid
    block &= ~seam
    stamp_body(w, bodies, 1, block, 0.9, vel=(-0.02, 0.01), spin=-0.001,
               subcell=(-0.1875, 0.0625), mobility=(0.5, 0.01, 0.002, 0.45, -0.003, 0.02), mobility_at=0)
    stamp_body(w, bodies, 2, box(width // 2 + 14, height - 5, 10, 4), 7.8, flags=abi.BF_ALIVE | abi.BF_HELD | abi.BF_WET)
    stamp_body(w, bodies, 3, box(width // 6 + 4, height - 12, 4, 4), 0.6, flags=abi.BF_ALIVE | abi.BF_NEW)
    stamp_body(w, bodies, 4, box(width - 14, surface + 4, 3, 5), 0.6, flags=0)
    # a hull: a floor 10 wide and sides 5 high, its hold 8 x 4 over the floor
    hx, hy = width // 2 - 6, surface - 3
    hull = np.zeros((height, width), dtype=bool)
    hull[hy + 4, hx:hx + 10] = True
    hull[hy:hy + 4, hx] = hull[hy:hy + 4, hx + 9] = True
    assert not np.any(hull & used)
    used[hull] = True
    stamp_body(w, bodies, 5, hull, 0.6, vel=(0.01, -0.02), spin=0.001, subcell=(0.0625, 0.125))
    hold = np.zeros((height, width), dtype=bool)
    hold[hy:hy + 4, hx + 1:hx + 9] = True
    cargo = np.zeros_like(hold)
    cargo[hy + 3, hx + 2:hx + 4] = True  # sand on the hold's floor: the hull's cargo
    w.paint(cargo, abi.SAND)
    used[cargo] = True
    water = np.zeros((height, width), dtype=bool)
    water[surface:height - 1, 1:width - 1] = True
    water &= ~used
    vel = rng.normal(0.0, 0.3, (height, width, 2)).astype(np.float32)
    w.paint(water, liquid, vel=vel)
    w.config = dict(workload="bodies_tank", grid=f"{width}x{height}", seed=seed, earth_g=earth_g_cells())
    if stamps:
        bodies.swept = [(np.flatnonzero(hold.ravel()), 5, False), (np.flatnonzero(seam.ravel()), 1, True)]
    return w, bodies


def send_aside(world, bodies, frame):
    """What bodies.wgsl leaves for the liquid's next step where a body pushed
    particles aside: their cell's G_DEST says DEST_ASIDE and the cell they
    go to.  Cells of the water under the hull are sent into its hold (which
    syncParticles refuses: another body's cup) and beside it (which it
    takes)."""
    if not bodies.swept:
        return
    cc = world.counters_cells()
    hold = bodies.swept[0][0]
    rows = hold // world.W
    below = (rows.max() + 2) * world.W + (hold % world.W)
    for k, src in enumerate(below[:4]):
        dst = hold[k] if k % 2 == 0 else src + 3 * world.W
        cc[src, 4] = 0x80000000 | int(dst)
