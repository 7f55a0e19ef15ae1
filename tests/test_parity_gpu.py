"""Parity of the CUDA liquid step with the CPU oracle, through the C ABI.

Grid buffers (cells, counters, field, blocks, cg) must match bit for bit;
particles as per-cell multisets (their order within a cell's run is an
atomic's order, as in the reference, shaders/fluid.wgsl:3707).  Velocity and
pressure therefore agree far inside the 1e-5 relative-L2 bar; the test
states that bar too, for the record.
"""
import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

import json
import os

from .common import busy_world, compare_worlds, params, run_membership
from .golden.make_golden import CASES, world_digests

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5  # the velocity / pressure bar of the drop-in


def _gpu():
    from worldinagrain_b200 import fluid
    return fluid


def _oracle(world):
    from oracle.oracle import Oracle
    return Oracle(world, W.element_table())


def _rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def _advance(world, steps, flags=0, max_cycles=abi.FLUID_CYCLES):
    o = _oracle(world)
    for s in range(1, steps + 1):
        o.step(params(world, s), max_cycles=max_cycles, flags=flags)
    return o


def _sequence(levels, max_cycles, shifted):
    """encodeFluid's dispatches (js/sim.js:2486-2611) as (pass, level, cycle)."""
    seq = [(p, 0, 0) for p in ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER",
                               "SEAL_JOIN", "SEAL_ANCHOR", "CLASSIFY", "SET_FACES", "UNPRESS", "DIVERGENCE",
                               "CG_START", "CG_JOIN", "CG_ANCHOR", "CG_RESIDUAL", "CG_PREPARE")]
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
        seq += [(p, 0, cyc) for p in ("CG_RHO", "CG_BETA", "CG_DIRECTION", "CG_APPLY", "CG_ALPHA", "CG_UPDATE")]
    seq += [(p, 0, 0) for p in ("CG_FINISH", "PROJECT", "EXTRAPOLATE", "EXTRAPOLATE_FURTHER", "ADVECT",
                                "SORT_COUNT", "SCAN_BLOCKS", "SCAN_TOTALS", "SCAN_FINISH", "SCATTER",
                                "RASTER_CLAIMS", "RASTER", "UNPAINT")]
    return seq


@pytest.mark.parametrize("kind,steps", [("dam", 3), ("obstacles", 6)])
def test_each_pass_matches_oracle(kind, steps):
    """Each reference pass, from the same state, leaves the same buffers."""
    fluid = _gpu()
    world = W.small_world(48, 40, seed=5, kind=kind)
    _advance(world, steps)
    o = _oracle(world)
    g = fluid.LiquidStep(world.copy(), W.element_table())
    P = params(world, steps + 1)
    seq = _sequence(len(world.L["levels"]), 3, shifted=True)
    got = world.copy()
    labelling = False  # G_REGION holds union-find links from sealJoin until cgFinish
    for name, level, cycle in seq:
        if name == "SEAL_JOIN":
            labelling = True
        if name == "CG_FINISH":
            labelling = False
        g.upload(world)
        o.pass_(P, name, level, cycle)
        g.dispatch(P, name, level, cycle)
        g.download(got)
        diffs = compare_worlds(got, world, region_links=labelling)
        assert not diffs, f"pass {name} (level {level}, cycle {cycle}): " + "; ".join(diffs)
    g.close()


FORMS = {"plain": abi.STEP_PLAIN, "fast": 0, "persistent": abi.STEP_PERSISTENT}


@pytest.mark.parametrize("form", ["plain", "fast", "persistent"])
@pytest.mark.parametrize("kind", ["dam", "obstacles", "moving"])
def test_steps_match_oracle(kind, form):
    """Whole steps (the captured graph) from the first seeding on: grid
    buffers bit for bit (the fast form's solve scratch aside), particles as
    multisets, every step."""
    fluid = _gpu()
    world = W.small_world(40, 32, seed=3, kind=kind)
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    for s in range(1, 13):
        P = params(ref, s)
        o.step(P)
        g.step(P, flags=FORMS[form])
        st = g.stats()
        g.download(got)
        diffs = compare_worlds(got, ref, scratch=form != "plain")
        assert not diffs, f"step {s}: " + "; ".join(diffs)
        assert run_membership(got)
        assert st.particles == int(ref.sorted[0])
        # the drop-in's numeric bar, stated: pressure and face velocity
        assert _rel_l2(got.pressure(), ref.pressure()) <= REL_L2
    g.close()


@pytest.mark.parametrize("form", ["plain", "fast", "persistent"])
@pytest.mark.parametrize("flags", [abi.STEP_TOLERANCE, abi.STEP_TOLERANCE | abi.STEP_F64_DOTS])
def test_tolerance_forms_match_oracle(flags, form):
    """The 1e-6 relative-residual forms: same iterations, same buffers."""
    fluid = _gpu()
    world = W.dam_break(64, 64)
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    for s in range(1, 9):
        P = params(ref, s)
        so = o.step(P, max_cycles=48, flags=flags, tolerance=1e-6)
        g.step(P, max_cycles=48, flags=flags | FORMS[form], tolerance=1e-6)
        sg = g.stats()
        g.download(got)
        diffs = compare_worlds(got, ref, scratch=form != "plain")
        assert not diffs, f"step {s}: " + "; ".join(diffs)
        assert sg.cycles == so.cycles
        assert sg.rel_residual <= 1e-6
        assert abs(sg.rel_residual - so.rel_residual) <= 1e-12 * max(1.0, so.rel_residual)
    g.close()


def test_coincident_particles_pushed_apart_alike():
    """Particles on one point (apart's pairWay, fluid.wgsl:703-707) are parted
    the same way on both sides."""
    fluid = _gpu()
    world = W.small_world(32, 32, seed=9, kind="dam")
    _advance(world, 2)
    m = world.sorted[4:].reshape(3, world.cap, 4)[0]
    cc = world.counters_cells()
    # put the second particle of every busy cell on its first's point
    starts = cc[:, 3][cc[:, 2] >= 2]
    m[starts + 1, :2] = m[starts, :2]
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    P = params(ref, 3)
    o.step(P)
    g.step(P)
    g.download(got)
    diffs = compare_worlds(got, ref, scratch=True)
    assert not diffs, "; ".join(diffs)
    g.close()


@pytest.mark.parametrize("form", ["fast", "persistent"])
@pytest.mark.parametrize("size,seed", [((256, 256), 1), ((200, 136), 4), ((131, 97), 6)])
def test_fast_form_matches_oracle_on_larger_worlds(size, seed, form):
    """The fast form on worlds whose levels go down through the per-level
    kernels into the one-CTA coarse kernel, world sides not multiples of 8
    included: several steps with the 1e-6 form, against the oracle."""
    fluid = _gpu()
    if size == (256, 256):
        world = W.dam_break(*size, seed=seed)
    else:
        world = W.small_world(*size, seed=seed, kind="obstacles")
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    flags = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
    for s in range(1, 5):
        P = params(ref, s)
        so = o.step(P, max_cycles=64, flags=flags, tolerance=1e-6)
        g.step(P, max_cycles=64, flags=flags | FORMS[form], tolerance=1e-6)
        sg = g.stats()
        g.download(got)
        diffs = compare_worlds(got, ref, scratch=True)
        assert not diffs, f"step {s}: " + "; ".join(diffs)
        assert sg.cycles == so.cycles
    g.close()


@pytest.mark.parametrize("form", ["fast", "persistent"])
def test_fast_profile_matches_graph(form):
    """The profiled (eagerly launched) fast step leaves what the graph leaves."""
    fluid = _gpu()
    world = W.small_world(48, 40, seed=2, kind="obstacles")
    a = fluid.LiquidStep(world.copy(), W.element_table())
    b = fluid.LiquidStep(world.copy(), W.element_table())
    wa, wb = world.copy(), world.copy()
    for s in range(1, 5):
        P = params(world, s)
        a.step(P, flags=abi.STEP_TOLERANCE | FORMS[form], tolerance=1e-6, max_cycles=40)
        prof = b.step_profile(P, flags=abi.STEP_TOLERANCE | FORMS[form], tolerance=1e-6, max_cycles=40)
        assert ("F_UPDATE" if form == "fast" else "F_SOLVE") in prof
        sa, sb = a.stats(), b.stats()
        assert sa.cycles == sb.cycles and sa.launches == sb.launches
        a.download(wa)
        b.download(wb)
        diffs = compare_worlds(wa, wb, scratch=True)
        assert not diffs, f"step {s}: " + "; ".join(diffs)
    a.close()
    b.close()


@pytest.mark.parametrize("form", ["plain", "fast", "persistent"])
@pytest.mark.parametrize("case", [c[0] for c in CASES])
def test_gpu_matches_golden_fixtures(case, form):
    """The committed fixtures (the oracle's digests, tests/golden): the
    plain form's every buffer, the fast forms' observable ones."""
    fluid = _gpu()
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "oracle_steps.json")) as f:
        want = json.load(f)[case]["steps"]
    name, builder, flags, max_cycles, record = next(c for c in CASES if c[0] == case)
    world = builder()
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    for s in range(1, max(record) + 1):
        P = W.make_params(world, frame=s, seed=0x1234, earth_g=world.config["earth_g"])
        g.step(P, max_cycles=max_cycles, flags=flags | FORMS[form], tolerance=1e-6)
        st = g.stats()
        if str(s) in want:
            g.download(got)
            d = world_digests(got)
            w = want[str(s)]
            keys = ["cells", "blocks", "sorted", "parts", "sorted_count", "parts_count"]
            keys += ["counters", "field", "cg"] if form == "plain" else ["counters_observable", "field_observable"]
            for k in keys:
                assert d[k] == w[k], f"{case} step {s} {k}"
            assert st.cycles == w["cycles"]
    g.close()


@pytest.mark.parametrize("form", ["plain", "fast"])
def test_two_liquids_with_viscosity(form):
    """Water and a viscous liquid: viscosity's sweeps and unpress
    (fluid.wgsl:3277-3466), two liquids' cells drawn by the most numerous
    (raster, fluid.wgsl:4029-4066), slip between them (fluid.wgsl:3605-3614)."""
    fluid = _gpu()
    world = W.two_liquids()
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    flags = abi.STEP_VISCOUS
    for s in range(1, 11):
        P = params(ref, s)
        so = o.step(P, flags=flags)
        g.step(P, flags=flags | FORMS[form])
        sg = g.stats()
        g.download(got)
        diffs = compare_worlds(got, ref, scratch=form != "plain")
        assert not diffs, f"step {s}: " + "; ".join(diffs)
        assert sg.count[abi.COUNT_VISCOUS] == so.count[abi.COUNT_VISCOUS] == 1
    g.close()


@pytest.mark.parametrize("k", [9, 120])  # sides 272 and 400 of the batched set, dam breaks
def test_fast_form_matches_oracle_on_batched_set_worlds(k):
    """Worlds of the batched set whose first two levels go through the tile
    kernels, the second with partial tiles at its edge: three steps of the
    1e-6 form against the oracle."""
    fluid = _gpu()
    world = W.multi_worlds(n=512, seed=2, only=[k])[0]
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    flags = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
    for s in range(1, 4):
        P = params(ref, s)
        so = o.step(P, max_cycles=64, flags=flags, tolerance=1e-6)
        g.step(P, max_cycles=64, flags=flags, tolerance=1e-6)
        sg = g.stats()
        g.download(got)
        diffs = compare_worlds(got, ref, scratch=True)
        assert not diffs, f"step {s}: " + "; ".join(diffs)
        assert sg.cycles == so.cycles
    g.close()
