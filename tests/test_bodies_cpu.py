"""The oracle's free-body coupling (fluid.wgsl:1181-1470, :2819-2845,
:2949-3218) on a tank with synthetic bodies, checked on the CPU by what the
coupled solve must do: the liquid beside a moving body is left as divergence
free as the rest (the body's faces moving with its push, PUSH_F), the bodies
the reference leaves out of the solve (just found, not alive) get nothing,
a held body's push is summed and it is marked wet, and no particle ends in a
body's cell."""
import json
import os

import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import params
from .golden.make_golden import BODY_CASES, run_body_case

HERE = os.path.dirname(os.path.abspath(__file__))

FLAGS = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS


def _oracle(world, bodies):
    from oracle.oracle import Oracle
    return Oracle(world, W.body_element_table(), bodies)


def _face_divergence(w):
    C, Wd, H, F = w.C, w.W, w.H, w.L["face_count"]
    faces = w.field.view(np.float32)[4 * 2 * C:4 * (2 * C + F)].reshape(F, 4)
    u = faces[:(Wd + 1) * H, 0].reshape(H, Wd + 1)
    v = faces[(Wd + 1) * H:, 0].reshape(H + 1, Wd)
    return (u[:, 1:] - u[:, :-1]) + (v[1:, :] - v[:-1, :])


def _solve_and_project(o, w, P, max_cycles=64):
    """The second half of a step, pass by pass, up to and including project."""
    for p in ["SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER", "SEAL_JOIN",
              "SEAL_ANCHOR", "CLASSIFY", "BODY_START", "BODY_LOADS", "SET_FACES", "UNPRESS", "DIVERGENCE",
              "CG_START", "CG_JOIN", "CG_ANCHOR", "CG_BODY_X", "CG_RESIDUAL", "CG_PREPARE"]:
        o.pass_(P, p)
    levels = len(w.L["levels"])
    sh = True
    for cyc in range(max_cycles):
        for p in ("RELAX_RIMS", "RELAX_SHIFTED" if sh else "RELAX"):
            o.pass_(P, p, 0, cyc)
        sh = not sh
        for l in range(1, levels + 1):
            o.pass_(P, "RESTRICT", l, cyc)
            if l < levels:
                o.pass_(P, "SMOOTH_RED", l, cyc)
                o.pass_(P, "SMOOTH_BLACK", l, cyc)
        o.pass_(P, "SOLVE", levels, cyc)
        for l in range(levels - 1, 0, -1):
            for p in ("PROLONG", "SMOOTH_RED", "SMOOTH_BLACK"):
                o.pass_(P, p, l, cyc)
        for p in ("PROLONG_FINE", "RELAX_RIMS", "RELAX_SHIFTED" if sh else "RELAX"):
            o.pass_(P, p, 0, cyc)
        sh = not sh
        for p in ("CG_RHO", "CG_BETA", "CG_DIRECTION", "CG_BODY_P", "CG_APPLY", "CG_ALPHA", "CG_UPDATE"):
            o.pass_(P, p, 0, cyc)
    o.pass_(P, "CG_FINISH")
    o.pass_(P, "CG_BODY_F")
    before = _face_divergence(w)
    o.pass_(P, "PROJECT")
    return before, _face_divergence(w)


def test_coupled_projection_leaves_the_liquid_beside_bodies_divergence_free():
    """The projection moves the bodies' faces with their push (PUSH_F), so a
    liquid cell beside a body is left with the solve's residual, as any
    other is."""
    w, bodies = W.bodies_world()
    o = _oracle(w, bodies)
    bodies.stamp_step(0)
    o.step(params(w, 1), max_cycles=64, flags=FLAGS, tolerance=1e-6)
    bodies.stamp_step(1)
    before, after = _solve_and_project(o, w, params(w, 2))
    rho = w.field_cells()[:, 0, 2].reshape(w.H, w.W)
    rigid = w.field_cells()[:, 1, 2].reshape(w.H, w.W) < -0.5
    near = np.zeros_like(rigid)
    near[:, 1:] |= rigid[:, :-1]
    near[:, :-1] |= rigid[:, 1:]
    near[1:, :] |= rigid[:-1, :]
    near[:-1, :] |= rigid[1:, :]
    liquid = rho > 0
    assert np.any(liquid & near)
    # the passes stop on the reference's rule, max|r| < 1e-2 (fluid.wgsl:2223-2226),
    # and what the projection leaves of a liquid cell's divergence is its -r:
    # beside the bodies as elsewhere, under that bound
    beside = np.abs(after[liquid & near]).max()
    elsewhere = np.abs(after[liquid & ~near]).max()
    assert beside < 1e-2 and elsewhere < 1e-2, (beside, elsewhere)
    assert beside < 0.1 * np.abs(before[liquid & near]).max()


@pytest.mark.parametrize("liquid,flags", [(abi.WATER, FLAGS), (W.MUD, FLAGS | abi.STEP_VISCOUS), (abi.WATER, 0)])
def test_bodies_in_and_out_of_the_solve(liquid, flags):
    w, bodies = W.bodies_world(liquid=liquid)
    o = _oracle(w, bodies)
    for s in range(1, 4):
        bodies.stamp_step(s - 1)
        W.send_aside(w, bodies, s)
        st = o.step(params(w, s), max_cycles=64, flags=flags, tolerance=1e-6)
        if flags & abi.STEP_TOLERANCE:
            assert st.rel_residual <= 1e-6
    drift_z = w.field_cells()[:, 1, 2]
    # the free bodies and the held one are in the solve, classified by slot
    # (fluid.wgsl:1657-1661): the block with its seam, the hull with its cargo
    for b, cells in ((0, 42), (1, 35 + 1), (5, 18 + 2)):
        assert int(np.sum(drift_z == np.float32(-1.0 - b))) == cells
    assert int(np.sum(drift_z == np.float32(-1.0 - (2 + abi.MAX_BODIES)))) == 40
    for b in (0, 1, 2, 5):
        assert np.any(bodies.liquid(b)[:3] != 0), b
    assert bodies.liquid(2)[3] & 0x80000000  # held and by the liquid: wet (LIQUID_WET)
    for b in (3, 4):  # just found, not alive: walls standing still, nothing done to them
        assert not np.any(bodies.liquid(b)), b
    pushes = bodies.pushes.reshape(abi.MAX_BODIES, 6, 6)
    assert np.any(pushes[0, 4] != 0)  # the pressure at the plank's surface as posed (PUSH_SURFACE)
    if flags & abi.STEP_VISCOUS:
        assert np.any(pushes[0, 5] != 0)  # the viscous liquid's drag (PUSH_DRAG)
    # particles stop at a body's cells as at any solid
    motion, _, _ = w.particles("sorted")
    cx = np.clip(np.floor(motion[:, 0]).astype(int), 0, w.W - 1)
    cy = np.clip(np.floor(motion[:, 1]).astype(int), 0, w.H - 1)
    kinds = w.cell_view()[cy, cx, 0] & 0xff
    assert not np.any(kinds == W.WOOD)


@pytest.mark.parametrize("case", [c[0] for c in BODY_CASES])
def test_oracle_with_bodies_matches_golden_fixtures(case):
    """The oracle's steps of the body tank against its committed digests
    (grid buffers, particles, body table, push sums)."""
    with open(os.path.join(HERE, "golden", "bodies_steps.json")) as f:
        fixture = json.load(f)[case]
    _, liquid, flags, max_cycles, record = next(c for c in BODY_CASES if c[0] == case)
    assert run_body_case(liquid, flags, max_cycles, record) == fixture["steps"]


def test_cup_and_seam_only_with_the_stamps():
    """Without the swept stamps (binding 14 unbound) the block's seam is the
    liquid's and the hull's sand is plain powder, a wall of no body."""
    w, bodies = W.bodies_world(stamps=False)
    o = _oracle(w, bodies)
    o.step(params(w, 1), max_cycles=64, flags=FLAGS, tolerance=1e-6)
    drift_z = w.field_cells()[:, 1, 2]
    assert int(np.sum(drift_z == np.float32(-2.0))) == 35
    assert int(np.sum(drift_z == np.float32(-6.0))) == 18


@pytest.mark.parametrize("liquid", ["water", "mud"])
def test_coupled_fp32_solve_reaches_the_fp64_solution_of_the_assembled_system(liquid):
    """The FP32 step's pressure (the coupling applied as the reference does,
    through the push sums and couplingAt) against an FP64 CG of the same
    system assembled on its own, L + J^T G J (the oracle's F64System): within
    the 1e-6 solve's error; and far from the FP64 solution of L alone, the
    bodies then walls that move but do not give way."""
    mud = liquid == "mud"
    w, bodies = W.bodies_world(liquid=W.MUD if mud else abi.WATER)
    flags = FLAGS | (abi.STEP_VISCOUS if mud else 0)
    o = _oracle(w, bodies)
    for s in (1, 2):
        bodies.stamp_step(s - 1)
        W.send_aside(w, bodies, s)
        o.step(params(w, s), max_cycles=64, flags=flags, tolerance=1e-6)
    bodies.stamp_step(2)
    P = params(w, 3)
    probe, probe_b = w.copy(), bodies.copy()
    po = _oracle(probe, probe_b)
    pre = ["SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER", "SEAL_JOIN",
           "SEAL_ANCHOR", "CLASSIFY", "BODY_START", "BODY_LOADS", "SET_FACES", "UNPRESS"]
    if mud:  # the sweeps' passes, then the drag, as a viscous step runs them
        pre += ["VISCOSITY_RED", "VISCOSITY_BLACK"] * 8 + ["UNPRESS", "BODY_DRAG", "BODY_FACES"]
        pre.remove("UNPRESS")
    pre += ["DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR"]
    for name in pre:
        po.pass_(P, name)
    x64, _, rel = po.solve_f64(P, rel_tol=1e-12)
    assert rel <= 1e-12
    from oracle.oracle import Oracle
    xl, _, rel_l = Oracle(probe.copy(), W.body_element_table(), None).solve_f64(P, rel_tol=1e-12)
    assert rel_l <= 1e-12
    st = o.step(P, max_cycles=64, flags=flags | abi.STEP_SHIFTED_SET, tolerance=1e-6)
    assert st.rel_residual <= 1e-6
    fluid = probe.field_cells()[:, 0, 2] > 0
    p = w.field_cells()[:, 0, 0][fluid].astype(np.float64)
    err = np.linalg.norm(p - x64[fluid]) / np.linalg.norm(x64[fluid])
    apart = np.linalg.norm(xl[fluid] - x64[fluid]) / np.linalg.norm(x64[fluid])
    print(f"\nbodies tank, {liquid}: pressure {err:.3e} relative L2 against the FP64 coupled solve "
          f"({apart:.3e} between the coupled and the uncoupled solves)")
    assert err < 1e-4, err
    assert apart > 100 * err, (apart, err)


def _still_tank(density, size=64, side=8):
    """A tank of still water, a quarter of it air, and a square body of the
    given density (water cells a cell) at rest at mid-depth."""
    w = W.World(size, size)
    bodies = W.Bodies(size, size)
    wall = np.zeros((size, size), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    w.paint(wall, abi.WALL)
    surface = size // 4
    body = np.zeros_like(wall)
    y0, x0 = (surface + size) // 2 - side // 2, size // 2 - side // 2
    body[y0:y0 + side, x0:x0 + side] = True
    W.stamp_body(w, bodies, 0, body, density)
    water = np.zeros_like(wall)
    water[surface:size - 1, 1:size - 1] = True
    w.paint(water & ~(wall | body), abi.WATER)
    w.config = dict(earth_g=W.earth_g_cells())
    return w, bodies


# The added mass of a square prism moving square to a face in still liquid,
# by potential flow: C_A = 1.51 on the area pi (b/2)^2, i.e. 1.19 rho b^2
# (the tabulated potential-flow coefficient of a square section, as in
# DNV-RP-C205's appendix A and Newman, Marine Hydrodynamics, 1977).
SQUARE_ADDED_MASS = 1.51 * np.pi / 4.0


@pytest.mark.parametrize("density", [1.0, 0.5, 2.0])
def test_a_body_released_in_still_water_moves_as_its_added_mass_has_it(density):
    """A physical anchor for the coupling: a square body at rest in still
    water, its first step.  Held by the liquid against the pull and free to
    give way, it takes the acceleration a = (rho_w - rho_b) V g / (m + m_A),
    m_A the liquid it sets moving; what the liquid does to it (its liquid
    words) is a - g along the pull: -g exactly at the liquid's own density
    (Archimedes: it neither rises nor sinks), and within 2% of the
    potential-flow added mass at half and twice it.  Nothing pushes it
    sideways or turns it."""
    w, bodies = _still_tank(density)
    o = _oracle(w, bodies)
    st = o.step(params(w, 1), max_cycles=64, flags=FLAGS, tolerance=1e-6)
    assert st.rel_residual <= 1e-6
    g = w.config["earth_g"]
    dv = bodies.liquid(0)[:3].view(np.int32).astype(np.float64) / abi.RIGID_FIX
    expected = -1.0 - (1.0 - density) / (density + SQUARE_ADDED_MASS)
    print(f"\ndensity {density}: liquid's dv_y {dv[1] / g:+.4f} g, potential flow {expected:+.4f} g")
    assert abs(dv[1] / g - expected) <= 0.02 * abs(expected), (dv[1] / g, expected)
    if density == 1.0:
        assert abs(dv[1] / g + 1.0) < 1e-3
    assert abs(dv[0]) < 1e-3 * g and abs(dv[2]) < 1e-3 * g


@pytest.mark.parametrize("density", [7.8, 2.0])
def test_a_held_block_on_the_floor_is_lifted_as_archimedes_has_it(density):
    """A held block resting on the floor of a still tank (heldPush, with
    seepAt finding the liquid's pressure beside it for the faces it rests
    on, fluid.wgsl:2977-3031): the liquid's push on it is Archimedes' lift,
    -g rho_w / rho_b along the pull, each step, within 0.5%, and turns it
    not at all."""
    size, side = 64, 8
    w = W.World(size, size)
    bodies = W.Bodies(size, size)
    wall = np.zeros((size, size), dtype=bool)
    wall[-1, :] = True
    wall[:, 0] = wall[:, -1] = True
    w.paint(wall, abi.WALL)
    block = np.zeros_like(wall)
    block[size - 1 - side:size - 1, size // 2 - side // 2:size // 2 + side // 2] = True
    W.stamp_body(w, bodies, 0, block, density, flags=abi.BF_ALIVE | abi.BF_HELD | abi.BF_WET)
    water = np.zeros_like(wall)
    water[size // 4:size - 1, 1:size - 1] = True
    w.paint(water & ~(wall | block), abi.WATER)
    w.config = dict(earth_g=W.earth_g_cells())
    o = _oracle(w, bodies)
    g = w.config["earth_g"]
    before = np.zeros(3)
    for s in range(1, 4):
        o.step(params(w, s), max_cycles=64, flags=FLAGS, tolerance=1e-6)
        now = bodies.liquid(0)[:3].view(np.int32).astype(np.float64) / abi.RIGID_FIX
        dv, before = now - before, now
        assert abs(dv[1] / g + 1.0 / density) <= 0.005 / density, (s, dv[1] / g)
        assert abs(dv[2]) < 1e-3 * g
    assert bodies.liquid(0)[3] & 0x80000000  # by the liquid: wet


def test_two_word_push_sums_are_exact_and_order_free():
    """The pushes' sums (common.wgsl:1378-1412): each value split into two
    words of 2^-24 units, the low added with its carry into the high, as the
    atomics add them.  In any order the words come out the same, also past
    2^31 units (|x| >= 128, which a large body in deep water reaches), and
    read back they are the sum of the rounded values."""
    from oracle.oracle import exact_parts, exact_value
    rng = np.random.default_rng(7)
    x = np.concatenate([rng.normal(0.0, 1e-3, 200), rng.normal(0.0, 30.0, 200), rng.uniform(-3e3, 3e3, 50)])
    x = x.astype(np.float32)
    parts = [exact_parts(float(v)) for v in x]
    assert any(abs(float(v)) >= 128.0 for v in x)
    units = [int(np.round(np.float64(v) * 16777216.0)) for v in x]
    for (lo, hi), u in zip(parts, units):  # each part pair is its value's units, two's complement
        assert ((hi << 32) | lo) == u % (1 << 64)
    totals = set()
    for _ in range(5):
        lo_sum = hi_sum = 0
        for k in rng.permutation(len(parts)):
            lo, hi = parts[k]
            old = lo_sum
            lo_sum = (old + lo) & 0xFFFFFFFF
            hi_sum = (hi_sum + hi + (1 if lo_sum < old else 0)) & 0xFFFFFFFF
        totals.add((lo_sum, hi_sum))
    assert len(totals) == 1
    lo_sum, hi_sum = totals.pop()
    want = sum(units) / 16777216.0
    assert abs(exact_value(lo_sum, hi_sum) - want) <= 1e-6 * max(1.0, abs(want))
