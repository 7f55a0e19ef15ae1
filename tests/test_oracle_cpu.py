"""The CPU oracle (oracle/wig_oracle.cpp) on its own: the invariants the
reference's scenes state, integer invariants of the splat, the FP64 solve,
determinism, and the committed golden fixtures.  No GPU."""
import json
import math
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, sincos
from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import params
from .golden.make_golden import CASES, world_digests

HERE = os.path.dirname(os.path.abspath(__file__))


def _run(world, steps, flags=0, max_cycles=16, tol=1e-6):
    o = Oracle(world, W.element_table())
    stats = []
    for s in range(1, steps + 1):
        stats.append(o.step(params(world, s), max_cycles=max_cycles, flags=flags, tolerance=tol))
    return o, stats


def test_own_sincos_matches_numpy():
    for a in np.linspace(0.0, 2 * math.pi, 2001, endpoint=False):
        s, c = sincos(float(np.float32(a)))
        assert abs(s - math.sin(np.float32(a))) < 2e-6
        assert abs(c - math.cos(np.float32(a))) < 2e-6


def test_dam_break_loses_no_particle():
    """js/scenes.js:1089-1090, `dam`: "Not a drop is lost"."""
    world = W.dam_break(64, 64)
    n0 = None
    o = Oracle(world, W.element_table())
    for s in range(1, 41):
        st = o.step(params(world, s))
        if n0 is None:
            n0 = st.particles
            water = int(np.sum(world.cell_view()[..., 0] & 0xff == abi.WATER))
            assert n0 == 4 * water
        assert st.particles == n0
        m, _, _ = world.particles()
        assert np.all(np.isfinite(m))
        # every particle inside the world and out of the walls' cells
        cx = np.floor(m[:, 0]).astype(int)
        cy = np.floor(m[:, 1]).astype(int)
        assert np.all((cx >= 1) & (cx < 63) & (cy >= 1) & (cy < 63))


def test_still_tank_pressure_grows_with_depth():
    """js/scenes.js:1085-1086, `still-tank`: it comes to rest, its pressure
    growing with depth (columnWeight, fluid.wgsl:1566-1575: rho g (depth + 1/2))."""
    world = W.World(32, 40)
    wall = np.zeros((40, 32), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    world.paint(wall, abi.WALL)
    water = np.zeros((40, 32), dtype=bool)
    water[20:39, 1:31] = True
    world.paint(water, abi.WATER)
    world.config = {"earth_g": W.earth_g_cells()}
    g = world.config["earth_g"]
    _run(world, 60, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, max_cycles=48)
    p = world.pressure()
    m, _, _ = world.particles()
    assert np.abs(m[:, 2:]).max() < 0.05 * g * 60  # far below free fall over the run
    col = p[24:38, 15]
    assert np.all(np.diff(col) > 0)  # deeper, higher
    slope = np.mean(np.diff(col))
    assert abs(slope - g) < 0.1 * g


def test_splat_integer_invariants():
    """gather's fixed-point sums (fluid.wgsl:1000-1087): a cell's count and
    mass are its particles', water's density 1 at 20 C a unit of 2^16 each."""
    world = W.small_world(40, 32, seed=3, kind="obstacles")
    o = Oracle(world, W.element_table())
    for s in range(1, 4):
        o.step(params(world, s))
    P = params(world, 4)
    for name in ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER"):
        o.pass_(P, name)
    cc = world.counters_cells()
    n = world.particle_count("parts")
    assert int(cc[:, 0].sum()) == n
    assert np.array_equal(cc[:, 7].astype(np.int64), cc[:, 0].astype(np.int64) * 65536)
    # each particle's four density shares sum to 2^16 (up to rounding of each)
    assert abs(int(cc[:, 6].astype(np.int64).sum()) - n * 65536) <= 4 * n


def test_oracle_is_deterministic():
    a = W.small_world(40, 32, seed=3, kind="moving")
    b = a.copy()
    _run(a, 5)
    _run(b, 5)
    for name in abi.BUFFER_NAMES:
        assert np.array_equal(getattr(a, name), getattr(b, name)), name


def test_fp32_solve_against_fp64_solve():
    """The oracle's FP32 CG (1e-6 form) against an FP64 solve of the same
    operator at 1e-12: the pressure's relative L2 error."""
    world = W.dam_break(64, 64)
    o, _ = _run(world, 3, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, max_cycles=48)
    P = params(world, 4)
    seq = ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER", "SEAL_JOIN",
           "SEAL_ANCHOR", "CLASSIFY", "SET_FACES", "UNPRESS", "DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR")
    probe = world.copy()
    po = Oracle(probe, W.element_table())
    for name in seq:
        po.pass_(P, name)
    x64, it, rel = po.solve_f64(P, rel_tol=1e-12)
    assert rel <= 1e-12
    o.step(P, max_cycles=48, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, tolerance=1e-6)
    x32 = world.field_cells()[:, 0, 0].astype(np.float64)
    fluid = world.field_cells()[:, 0, 2] > 0
    err = np.linalg.norm(x32[fluid] - x64[fluid]) / np.linalg.norm(x64[fluid])
    assert err < 1e-4, err
    true_rel = po.true_residual(P, world.field_cells()[:, 0, 0])
    assert true_rel < 1e-3


@pytest.mark.parametrize("builder", [lambda: W.dam_break(128, 128), lambda: W.small_world(96, 80, seed=4, kind="obstacles")])
def test_multigrid_fp64_solve_matches_jacobi_fp64_solve(builder):
    """The FP64 solve preconditioned by the oracle's V-cycle (for the large
    worlds) reaches the same solution as the Jacobi-preconditioned one, in
    far fewer iterations."""
    world = builder()
    _run(world, 3, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, max_cycles=48)
    P = params(world, 4)
    seq = ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER", "SEAL_JOIN",
           "SEAL_ANCHOR", "CLASSIFY", "SET_FACES", "UNPRESS", "DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR")
    po = Oracle(world, W.element_table())
    for name in seq:
        po.pass_(P, name)
    xj, itj, relj = Oracle(world.copy(), W.element_table()).solve_f64(P, rel_tol=1e-12)
    xm, itm, relm = Oracle(world.copy(), W.element_table()).solve_f64(P, rel_tol=1e-12, multigrid=True)
    assert relj <= 1e-12 and relm <= 1e-12
    assert itm < itj / 4, (itm, itj)
    assert np.linalg.norm(xm - xj) <= 1e-9 * np.linalg.norm(xj)


def test_min_max_take_wgsl_nan_rule():
    """f32 min and max in the oracle follow WGSL's builtins (a NaN operand
    gives the other one), as the GPU's fminf and fmaxf do, so non-finite
    particles step alike on both: checked through the sub-step count of a
    travel with one NaN component, which a std::max would make NaN."""
    world = W.small_world(32, 32, seed=7, kind="dam")
    _run(world, 2)
    m = world.sorted[4:].reshape(3, world.cap, 4)[0].view(np.float32)
    n = int(world.sorted[0])
    m[n // 2, 2] = np.float32("nan")
    o = Oracle(world, W.element_table())
    o.step(params(world, 3))
    assert int(world.sorted[0]) > 0
    assert np.all(np.isfinite(world.pressure()))


@pytest.mark.parametrize("case", [c[0] for c in CASES])
def test_oracle_matches_golden_fixtures(case):
    with open(os.path.join(HERE, "golden", "oracle_steps.json")) as f:
        fixtures = json.load(f)
    name, builder, flags, max_cycles, record = next(c for c in CASES if c[0] == case)
    world = builder()
    o = Oracle(world, W.element_table())
    want = fixtures[case]["steps"]
    for s in range(1, max(record) + 1):
        P = W.make_params(world, frame=s, seed=0x1234, earth_g=world.config["earth_g"])
        st = o.step(P, max_cycles=max_cycles, flags=flags, tolerance=1e-6)
        if str(s) in want:
            got = world_digests(world)
            got["cycles"] = int(st.cycles)
            assert got == want[str(s)], f"{case} step {s}"


def test_free_fall_gains_g_each_step():
    """A blob of water in open air falls freely: each step's pull on its
    faces (setFace, fluid.wgsl:1966-1973) leaves no divergence for the
    pressure to take back, so its particles' mean velocity is s g after s
    steps, within 0.2%, and nothing pushes them sideways."""
    world = W.World(48, 128)
    blob = np.zeros((128, 48), dtype=bool)
    blob[8:20, 16:32] = True
    world.paint(blob, abi.WATER)
    world.config = {"earth_g": W.earth_g_cells()}
    g = world.config["earth_g"]
    o = Oracle(world, W.element_table())
    for s in range(1, 41):
        o.step(params(world, s), max_cycles=64, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, tolerance=1e-6)
        m, _, _ = world.particles()
        assert len(m) == 12 * 16 * 4
        assert abs(m[:, 3].mean() / (s * g) - 1.0) < 2e-3, s
        assert abs(m[:, 2].mean()) < 1e-2 * g


def test_slot_in_a_tank_floor_discharges_as_kirchhoff_has_it():
    """Torricelli through a slot 4 cells wide in the floor of a tank 80 cells
    deep: the discharge a step, over the slot's width, is C sqrt(2 g h),
    with C the contraction of a jet from a slot in a wide wall, pi / (pi + 2)
    = 0.611 (Kirchhoff's free-streamline solution), within 12% (measured
    0.58)."""
    H, Wd, floor = 120, 64, 100
    world = W.World(Wd, H)
    wall = np.zeros((H, Wd), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    wall[floor, 1:Wd - 1] = True
    wall[floor, Wd // 2 - 2:Wd // 2 + 2] = False
    world.paint(wall, abi.WALL)
    water = np.zeros((H, Wd), dtype=bool)
    water[20:floor, 1:Wd - 1] = True
    world.paint(water, abi.WATER)
    world.config = {"earth_g": W.earth_g_cells()}
    g = world.config["earth_g"]
    o = Oracle(world, W.element_table())
    held = {}
    for s in range(1, 141):
        o.step(params(world, s), max_cycles=64, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, tolerance=1e-6)
        if s in (60, 140):
            m, _, _ = world.particles()
            inside = m[m[:, 1] < floor]
            held[s] = (len(inside), floor - np.percentile(inside[:, 1], 0.5))
    q = (held[60][0] - held[140][0]) / 80.0 / 4.0  # cells of liquid a step, 4 particles a cell
    h = 0.5 * (held[60][1] + held[140][1])
    c = q / 4.0 / math.sqrt(2.0 * g * h)
    kirchhoff = math.pi / (math.pi + 2.0)
    assert abs(c - kirchhoff) <= 0.12 * kirchhoff, c


def _poiseuille_startup(t, width, nu):
    """The centre speed of plane Poiseuille flow started from rest, over its
    steady g W^2 / (8 nu): 1 - (32 / pi^3) sum over odd n of (-1)^((n-1)/2)
    exp(-n^2 pi^2 nu t / W^2) / n^3 (the series solution of the diffusion of
    momentum from no-slip walls)."""
    s = 0.0
    for n in range(1, 200, 2):
        s += (-1) ** ((n - 1) // 2) * math.exp(-(n * math.pi) ** 2 * nu * t / width ** 2) / n ** 3
    return 1.0 - 32.0 / math.pi ** 3 * s


def test_viscous_liquid_drains_down_a_channel_as_poiseuille_flow():
    """A viscous liquid (this table's mud, nu = 0.8 cells^2 a step) falling
    down a vertical channel 20 cells wide and out of its open end: the
    viscosity's sweeps with no slip at the walls (viscousFace,
    fluid.wgsl:3347-3403) give the parabola u = g x (W - x) / (2 nu) across
    it, within 3% in shape, and its centre speed follows the start-up of
    Poiseuille flow from rest within 3% after 120 and 200 steps."""
    Wd, H, x0, x1, bottom = 64, 200, 23, 43, 150
    world = W.World(Wd, H)
    wall = np.zeros((H, Wd), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    wall[:bottom, x0 - 1] = True
    wall[:bottom, x1] = True
    world.paint(wall, abi.WALL)
    mud = np.zeros((H, Wd), dtype=bool)
    mud[10:140, x0:x1] = True
    world.paint(mud, W.MUD)
    world.config = {"earth_g": W.earth_g_cells()}
    g = world.config["earth_g"]
    elems = W.element_table()
    nu = elems[W.MUD].viscosity
    o = Oracle(world, elems)
    xc = np.arange(x0, x1) + 0.5
    steady = g / (2.0 * nu) * (xc - x0) * (x1 - xc)
    for s in range(1, 201):
        o.step(params(world, s), max_cycles=64,
               flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS | abi.STEP_VISCOUS, tolerance=1e-6)
        if s in (120, 200):
            m, _, _ = world.particles()
            mid = m[(m[:, 1] > 60) & (m[:, 1] < 100)]
            cols = np.floor(mid[:, 0]).astype(int)
            prof = np.array([mid[cols == c, 3].mean() for c in range(x0, x1)])
            shape = np.linalg.norm(prof / prof.max() - steady / steady.max()) / np.linalg.norm(steady / steady.max())
            ratio = prof.max() / steady.max()
            expected = _poiseuille_startup(s, x1 - x0, nu)
            assert shape < 0.03, (s, shape)
            assert abs(ratio - expected) < 0.03 * expected, (s, ratio, expected)


def test_two_layers_at_rest_hold_each_its_own_hydrostatic_gradient():
    """Water resting on a denser liquid (this table's mud, 1.6 times water)
    stays at rest, and the pressure grows by rho g a cell of depth in each
    layer, water's 1.0 and mud's 1.6, within 1%."""
    world = W.World(32, 48)
    wall = np.zeros((48, 32), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    world.paint(wall, abi.WALL)
    water = np.zeros((48, 32), dtype=bool)
    water[12:28, 1:31] = True
    world.paint(water, abi.WATER)
    mud = np.zeros((48, 32), dtype=bool)
    mud[28:47, 1:31] = True
    world.paint(mud, W.MUD)
    world.config = {"earth_g": W.earth_g_cells()}
    g = world.config["earth_g"]
    elems = W.element_table()
    o = Oracle(world, elems)
    for s in range(1, 81):
        o.step(params(world, s), max_cycles=64,
               flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS | abi.STEP_VISCOUS, tolerance=1e-6)
    col = world.pressure()[:, 15]
    for rows, elem in ((slice(15, 26), abi.WATER), (slice(31, 45), W.MUD)):
        slope = np.mean(np.diff(col[rows])) / g
        rho = elems[elem].density / 100.0
        assert abs(slope - rho) < 0.01 * rho, (elem, slope)
    m, _, _ = world.particles()
    assert np.abs(m[:, 2:]).max() < 0.01 * 80 * g  # at rest: far below free fall over the run


def _inverted_tube(capped):
    """A tube 8 cells wide and 55 tall standing in a basin of water, full;
    capped: closed at its top (an inverted test tube), else open there."""
    Wd, H = 48, 80
    world = W.World(Wd, H)
    wall = np.zeros((H, Wd), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    if capped:
        wall[10, 19:29] = True
    wall[10:66, 19] = True
    wall[10:66, 28] = True
    world.paint(wall, abi.WALL)
    water = np.zeros((H, Wd), dtype=bool)
    water[11:66, 20:28] = True
    water[55:79, 1:47] = True
    world.paint(water & ~wall, abi.WATER)
    world.config = {"earth_g": W.earth_g_cells()}
    return world


@pytest.mark.parametrize("capped", [True, False])
def test_a_capped_tube_holds_its_water_up_and_an_open_one_drains(capped):
    """Space the liquid leaves with no way in for the air is a vacuum, and
    its suction holds the column (classify's sealed cells, sealJoin and
    sealAnchor, fluid.wgsl:1483-1560, :1591-1600): a tube closed at its top,
    standing full in a basin, keeps all its water over the basin's surface
    for 150 steps; open at its top, the same tube drains into the basin
    (more than 5% of its water gone)."""
    world = _inverted_tube(capped)
    o = Oracle(world, W.element_table())

    def in_tube():
        m, _, _ = world.particles()
        return m[(m[:, 0] > 20) & (m[:, 0] < 28) & (m[:, 1] < 55)]

    start = None
    for s in range(1, 151):
        o.step(params(world, s), max_cycles=64, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, tolerance=1e-6)
        if s == 1:  # seeded by the first step
            start = len(in_tube())
    assert start == 44 * 8 * 4  # the tube's rows over the basin's surface, 4 particles a cell
    left = in_tube()
    if capped:
        assert len(left) == start and left[:, 1].min() < 11.5
    else:
        assert len(left) < 0.95 * start


def test_a_spinning_disk_keeps_its_angular_momentum():
    """A disk of water spinning rigidly with no pull: the APIC transfers
    (gather's affine splat, advect's affine update, fluid.wgsl:1000-1087,
    :3616-3694) carry the rotation between particles and grid, so its
    angular momentum stays within 2% after 50 steps and 6% after 200
    (measured 1.0% and 4.1%: the reference damps the affine part a little a
    step, AFFINE_KEEP), while the disk spreads as it spins."""
    N, om = 64, 0.01
    world = W.World(N, N)
    yy, xx = np.mgrid[0:N, 0:N] + 0.5
    disk = (xx - N / 2) ** 2 + (yy - N / 2) ** 2 < 14 ** 2
    vel = np.zeros((N, N, 2), dtype=np.float32)
    vel[..., 0] = -om * (yy - N / 2)
    vel[..., 1] = om * (xx - N / 2)
    world.paint(disk, abi.WATER, vel=vel)
    o = Oracle(world, W.element_table())

    def angular_momentum():
        m, _, _ = world.particles()
        rx, ry = m[:, 0] - m[:, 0].mean(), m[:, 1] - m[:, 1].mean()
        return float(np.sum(rx * m[:, 3] - ry * m[:, 2]))

    held = {}
    for s in range(1, 201):
        o.step(W.make_params(world, frame=s, seed=2, earth_g=0.0), max_cycles=64,
               flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, tolerance=1e-6)
        if s in (1, 50, 200):
            held[s] = angular_momentum()
    assert held[1] > 0
    assert held[50] / held[1] > 0.98
    assert held[200] / held[1] > 0.94
