"""Parity of the CUDA liquid step with free bodies coupled into its solve
(A = L + J^T M^-1 J: fluid.wgsl:1181-1470, :2819-2845, :2949-3218; the
dispatches of js/sim.js:2499-2600) against the CPU oracle, through the C ABI
(wig_fluid_bind_bodies).  The tank holds synthetic bodies: a plank afloat,
moving and spinning with a sub-cell pose; a block under the water with a
contact mobility and a seam in its wall; a held, wet block on the floor; a
body just found; a slot not alive; and a hull whose cup (its swept stamps)
holds sand as cargo, with particles sent aside into and beside it.  Grid buffers, the body table (its liquid words) and the
push sums must match bit for bit, particles as multisets."""
import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import compare_worlds, diff_words, params, run_membership

pytestmark = pytest.mark.gpu

TOL = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS


def _oracle(world, bodies):
    from oracle.oracle import Oracle
    return Oracle(world, W.body_element_table(), bodies)


def _body_diffs(got, ref):
    out = []
    for name in ("motion", "pushes"):
        d = diff_words(getattr(got, name), getattr(ref, name), name)
        if d:
            out.append(d)
    return out


def _sequence(levels, max_cycles, shifted, drag=False):
    """encodeFluid's dispatches with the bodies' passes (js/sim.js:2486-2611);
    drag: the liquid's drag on the bodies after unpress (a viscous world's)."""
    seq = [(p, 0, 0) for p in ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER",
                               "SEAL_JOIN", "SEAL_ANCHOR", "CLASSIFY", "BODY_START", "BODY_LOADS", "SET_FACES",
                               "UNPRESS") + (("BODY_DRAG", "BODY_FACES") if drag else ()) +
           ("DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR", "CG_BODY_X", "CG_RESIDUAL", "CG_PREPARE")]
    sh = shifted
    for cyc in range(max_cycles):
        seq += [("RELAX_RIMS", 0, cyc), ("RELAX_SHIFTED" if sh else "RELAX", 0, cyc)]
        sh = not sh
        for l in range(1, levels + 1):
            seq.append(("RESTRICT", l, cyc))
            if l < levels:
                seq += [("SMOOTH_RED", l, cyc), ("SMOOTH_BLACK", l, cyc)]
        seq.append(("SOLVE", levels, cyc))
        for l in range(levels - 1, 0, -1):
            seq += [("PROLONG", l, cyc), ("SMOOTH_RED", l, cyc), ("SMOOTH_BLACK", l, cyc)]
        seq += [("PROLONG_FINE", 0, cyc), ("RELAX_RIMS", 0, cyc), ("RELAX_SHIFTED" if sh else "RELAX", 0, cyc)]
        sh = not sh
        seq += [(p, 0, cyc) for p in ("CG_RHO", "CG_BETA", "CG_DIRECTION", "CG_BODY_P", "CG_APPLY", "CG_ALPHA",
                                      "CG_UPDATE")]
    seq += [(p, 0, 0) for p in ("CG_FINISH", "CG_BODY_F", "PROJECT", "RIGIDIFY", "BODY_PUSH", "EXTRAPOLATE",
                                "EXTRAPOLATE_FURTHER", "ADVECT", "SORT_COUNT", "SCAN_BLOCKS", "SCAN_TOTALS",
                                "SCAN_FINISH", "SCATTER", "RASTER_CLAIMS", "RASTER", "UNPAINT")]
    return seq


@pytest.mark.parametrize("liquid", ["water", "mud"])
def test_each_pass_with_bodies_matches_oracle(liquid):
    """Each pass, the bodies' own among them, from the same state (a tank
    stepped twice) leaves the same buffers and body words."""
    from worldinagrain_b200 import fluid
    mud = liquid == "mud"
    world, bodies = W.bodies_world(liquid=W.MUD if mud else abi.WATER)
    o = _oracle(world, bodies)
    for s in (1, 2):
        bodies.stamp_step(s - 1)
        W.send_aside(world, bodies, s)
        o.step(params(world, s), max_cycles=64, flags=TOL | (abi.STEP_VISCOUS if mud else 0), tolerance=1e-6)
    bodies.stamp_step(2)
    W.send_aside(world, bodies, 3)
    g = fluid.LiquidStep(world.copy(), W.body_element_table())
    g.bind_bodies(bodies)
    P = params(world, 3)
    got, got_b = world.copy(), bodies.copy()
    labelling = False
    for name, level, cycle in _sequence(len(world.L["levels"]), 3, shifted=True, drag=mud):
        if name == "SEAL_JOIN":
            labelling = True
        if name == "CG_FINISH":
            labelling = False
        g.upload(world)
        g.upload_bodies(bodies)
        o.pass_(P, name, level, cycle)
        g.dispatch(P, name, level, cycle)
        g.download(got)
        g.download_bodies(got_b)
        diffs = compare_worlds(got, world, region_links=labelling) + _body_diffs(got_b, bodies)
        assert not diffs, f"pass {name} (level {level}, cycle {cycle}): " + "; ".join(diffs)
    g.close()


@pytest.mark.parametrize("case", ["water_tolerance", "water_default", "mud_viscous", "fast_flags"])
def test_steps_with_bodies_match_oracle(case):
    """Whole steps (the captured graph) with the bodies coupled, every step
    compared.  fast_flags asks for the fast form, which a world with bodies
    does not take: it steps the plain form's same bits."""
    from worldinagrain_b200 import fluid
    liquid, flags, cycles, steps = {
        "water_tolerance": (abi.WATER, TOL, 64, 6),
        "water_default": (abi.WATER, 0, abi.FLUID_CYCLES, 4),
        "mud_viscous": (W.MUD, TOL | abi.STEP_VISCOUS, 64, 4),
        "fast_flags": (abi.WATER, TOL, 64, 3),
    }[case]
    world, bodies = W.bodies_world(liquid=liquid)
    ref, ref_b = world.copy(), bodies.copy()
    o = _oracle(ref, ref_b)
    g = fluid.LiquidStep(world, W.body_element_table())
    g.bind_bodies(bodies)
    got, got_b = world.copy(), bodies.copy()
    gpu_flags = (flags | abi.STEP_MIXED) if case == "fast_flags" else (flags | abi.STEP_PLAIN)
    for s in range(1, steps + 1):
        P = params(ref, s)
        # what the bodies' pass would leave: this step's stamps, particles sent aside
        for wd, bd in ((ref, ref_b), (got, got_b)):
            bd.stamp_step(s - 1)
            W.send_aside(wd, bd, s)
        g.upload(got)
        g.upload_bodies(got_b)
        ost = o.step(P, max_cycles=cycles, flags=flags, tolerance=1e-6)
        g.step(P, max_cycles=cycles, flags=gpu_flags, tolerance=1e-6)
        st = g.stats(unconverged_ok=not (flags & abi.STEP_TOLERANCE))
        g.download(got)
        g.download_bodies(got_b)
        diffs = compare_worlds(got, ref) + _body_diffs(got_b, ref_b)
        assert not diffs, f"step {s}: " + "; ".join(diffs)
        assert run_membership(got)
        assert st.cycles == ost.cycles
        if flags & abi.STEP_TOLERANCE:
            assert st.rel_residual <= 1e-6
    for b in (0, 1, 2, 5):
        assert np.any(got_b.liquid(b)[:3] != 0)
    g.close()
