"""Parity with the oracle on the benchmark's own workloads, stepped as the
benchmark steps them: the same worlds and seeds, the 1e-6 relative-residual
form with FP64 dot products, max_cycles 64, the Params seed 2, and on a
single world the tiling parity fixed by the step's number.

- disks 1024x1024 (the bench's single world), fast form, three steps;
- dam 256x256, plain and fast forms, 24 steps;
- column 2048x2048 at 2 particles a cell: the first step of the plain and
  fast forms bit for bit, and after three steps every form's pressure and
  velocity error against an FP64 solve of the fourth step's system;
- twelve worlds spread over the 512-world batched set (sides 64 to 512,
  dams and columns), stepped as one batch under the launch shapes the
  bench's tuner picks: the fast form bit for bit over three steps, the
  mixed form's first step against an FP64 solve of each world.

Bit for bit means every grid word but the solve's scratch, particles as
per-cell multisets (tests/common.py), the same iteration counts and
residuals to 1e-12.  The mixed form rounds its multigrid words to binary16,
so it is held to the FP64 solve instead: its pressure and velocity errors
at most twice the FP32 form's plus 1e-5 (relative L2; the velocity's over
the velocity the projection acted on)."""
import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import compare_worlds, run_membership

pytestmark = pytest.mark.gpu

TOL = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
SEED = 2  # the bench's --seed, which also seeds each step's Params
PRE = ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER", "SEAL_JOIN",
       "SEAL_ANCHOR", "CLASSIFY", "SET_FACES", "UNPRESS", "DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR")
# the shapes the bench's autotuner picked for the 512-world set
BATCH_SHAPES = {"coarse_cells": 2048, "level_per_sm": 32, "cg_per_sm": 32, "relax_per_sm": 64}


def _params(world, step):
    return W.make_params(world, frame=step, seed=SEED, earth_g=world.config["earth_g"])


def _flags_of(step):
    # bench.py: the tiling parity follows the step's number
    return TOL | abi.STEP_SHIFTED_SET | (abi.STEP_SHIFTED_FIRST if step % 2 else 0)


def _oracle(world):
    from oracle.oracle import Oracle
    return Oracle(world, W.element_table())


def _same_step(got, ref, sg, so, scratch):
    diffs = compare_worlds(got, ref, scratch=scratch)
    assert not diffs, "; ".join(diffs)
    assert run_membership(got)
    assert sg.particles == int(ref.sorted[0])
    assert sg.cycles == so.cycles
    assert sg.rel_residual <= 1e-6
    assert abs(sg.rel_residual - so.rel_residual) <= 1e-12 * max(1.0, so.rel_residual)


def _faces(world):
    F = world.L["face_count"]
    return world.field[8 * world.C: 8 * world.C + 4 * F].reshape(F, 4)


def _fp64_system(world, P):
    """(probe: the world after the step's passes up to cgAnchor, the FP64
    pressure of the step's system to a 1e-12 relative residual)."""
    probe = world.copy()
    o = _oracle(probe)
    for name in PRE:
        o.pass_(P, name)
    scratch = probe.copy()
    x64, _, rel = _oracle(scratch).solve_f64(P, rel_tol=1e-12, max_iter=2000, multigrid=True)
    assert rel <= 1e-12
    return probe, x64


def _errors(probe, P, x64, stepped):
    """Relative L2 errors of a stepped world's pressure (liquid cells) and
    projected face velocities against the FP64 solve: the oracle's project
    pass run with each pressure on the probe."""
    fluid_ = probe.field_cells()[:, 0, 2] > 0
    p = stepped.field_cells()[:, 0, 0].copy()
    drift = stepped.field_cells()[:, 1, 0].copy()
    ep = np.linalg.norm(p[fluid_].astype(np.float64) - x64[fluid_]) / np.linalg.norm(x64[fluid_])

    def projected(pressure):
        q = probe.copy()
        fc = q.field_cells()
        fc[:, 0, 0] = pressure
        fc[:, 1, 0] = drift
        _oracle(q).pass_(P, "PROJECT")
        return _faces(q)

    ua = projected(p)
    ub = projected(np.where(fluid_, x64, p).astype(np.float32))
    on = ub[:, 2] == 2.0  # the faces the pass projected
    du = np.linalg.norm(ua[on, 0].astype(np.float64) - ub[on, 0])
    eu = du / np.linalg.norm(ub[on, 0].astype(np.float64))
    # the same gap over the velocity the projection acted on (the faces as
    # the step's passes before the solve left them): the measure that stays
    # meaningful where the liquid is at rest and the projected velocity is
    # all but zero
    ustar = _faces(probe)[on, 0].astype(np.float64)
    eu_star = du / max(np.linalg.norm(ustar), 1e-30)
    return float(ep), float(eu), ua[:, 0], on, float(eu_star)


def test_disks_1024_fast_form_matches_oracle():
    """The bench's single world, three steps of the fast form (with the
    single world's default launch shapes, the tuner's pick)."""
    from worldinagrain_b200 import fluid
    world = W.disks_world(1024, 1024, seed=SEED)
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    for s in range(1, 4):
        P = _params(ref, s)
        so = o.step(P, max_cycles=64, flags=_flags_of(s), tolerance=1e-6)
        g.step(P, max_cycles=64, flags=_flags_of(s), tolerance=1e-6)
        sg = g.stats()
        g.download(got)
        _same_step(got, ref, sg, so, scratch=True)
    g.close()


@pytest.mark.parametrize("form", ["plain", "fast"])
def test_dam_256_matches_oracle_over_24_steps(form):
    from worldinagrain_b200 import fluid
    world = W.dam_break(256, 256, seed=SEED)
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    extra = abi.STEP_PLAIN if form == "plain" else 0
    for s in range(1, 25):
        P = _params(ref, s)
        so = o.step(P, max_cycles=64, flags=_flags_of(s), tolerance=1e-6)
        g.step(P, max_cycles=64, flags=_flags_of(s) | extra, tolerance=1e-6)
        sg = g.stats()
        g.download(got)
        _same_step(got, ref, sg, so, scratch=form != "plain")
    g.close()


def test_column_2048_forms_match_oracle_and_fp64_solve():
    """Config 3's world: its first step, plain and fast bit for bit with the
    oracle; then, from the state after three steps (as the accuracy tests
    take it), every form's pressure and velocity against the FP64 solve of
    the fourth step's system, printed (pytest -s) and bounded.  The column
    is nearly at rest, so its velocity error is also given over the
    velocity the projection acted on."""
    from worldinagrain_b200 import fluid
    world = W.obstacle_column(2048, 2048)
    P = _params(world, 1)
    ref = world.copy()
    so = _oracle(ref).step(P, max_cycles=64, flags=_flags_of(1), tolerance=1e-6)
    for form, extra in (("plain", abi.STEP_PLAIN), ("fast", 0)):
        w = world.copy()
        g = fluid.LiquidStep(w, W.element_table())
        g.step(P, max_cycles=64, flags=_flags_of(1) | extra, tolerance=1e-6)
        sg = g.stats()
        g.download()
        _same_step(w, ref, sg, so, scratch=form != "plain")
        if form == "fast":
            # on to the third step (the fast form is the oracle's bits)
            for s in (2, 3):
                g.step(_params(w, s), max_cycles=64, flags=_flags_of(s), tolerance=1e-6)
                g.stats()
            w3 = g.download(w.copy())
        g.close()
    P4 = _params(w3, 4)
    probe, x64 = _fp64_system(w3, P4)
    out = {}
    for form, extra in (("plain", abi.STEP_PLAIN), ("fast", 0), ("mixed", abi.STEP_MIXED)):
        w = w3.copy()
        g = fluid.LiquidStep(w, W.element_table())
        g.step(P4, max_cycles=64, flags=_flags_of(4) | extra, tolerance=1e-6)
        sg = g.stats()
        g.download()
        g.close()
        assert sg.rel_residual <= 1e-6
        e = _errors(probe, P4, x64, w)
        out[form] = e
        print(f"\ncolumn 2048x2048 {form}: pressure {e[0]:.3e}, velocity {e[1]:.3e} relative L2 against the FP64 "
              f"solve ({e[4]:.3e} of the velocity projected); {sg.cycles} iterations, residual {sg.rel_residual:.2e}")
    assert out["plain"][0] == out["fast"][0]
    assert out["fast"][0] < 1e-3 and out["fast"][4] < 1e-3
    assert out["mixed"][0] <= 2 * out["fast"][0] + 1e-5
    assert out["mixed"][4] <= 2 * out["fast"][4] + 1e-5


def _batched_sample():
    """Twelve worlds at evenly spaced ranks of the 512-world set's sides:
    the smallest (64) to the largest (512), dams and columns."""
    specs = W.multi_world_specs(512, seed=SEED)
    order = sorted(range(512), key=lambda k: (specs[k][0], k))
    pick = [order[round(q * 511 / 11)] for q in range(12)]
    return pick, W.multi_worlds(n=512, seed=SEED, only=pick)


def test_batched_sample_fast_form_matches_oracle():
    from worldinagrain_b200 import fluid
    pick, worlds = _batched_sample()
    refs = [w.copy() for w in worlds]
    oracles = [_oracle(r) for r in refs]
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    for name, v in BATCH_SHAPES.items():
        b.set_launch(name, v)
    ids = list(range(len(mine)))
    for s in range(1, 4):
        so = [o.step(_params(r, s), max_cycles=64, flags=TOL, tolerance=1e-6) for o, r in zip(oracles, refs)]
        b.step(ids, [_params(w, s) for w in mine], max_cycles=64, flags=TOL, tolerance=1e-6)
        sg = b.stats(ids)
        for k, w in enumerate(mine):
            b.download(k)
            try:
                _same_step(w, refs[k], sg[k], so[k], scratch=True)
            except AssertionError as e:
                raise AssertionError(f"step {s}, world {pick[k]} (side {w.W}): {e}") from None
    b.close()


def test_batched_sample_mixed_form_against_fp64_solve():
    """The batched bench's form (mixed) on the sample, one step as a batch:
    each world's pressure and velocity against an FP64 solve of its system,
    beside the FP32 fast form's."""
    from worldinagrain_b200 import fluid
    pick, worlds = _batched_sample()
    ids = list(range(len(worlds)))
    stepped = {}
    for form, extra in (("fast", 0), ("mixed", abi.STEP_MIXED)):
        mine = [w.copy() for w in worlds]
        b = fluid.Batch(mine, W.element_table())
        for name, v in BATCH_SHAPES.items():
            b.set_launch(name, v)
        b.step(ids, [_params(w, 1) for w in mine], max_cycles=64, flags=TOL | extra, tolerance=1e-6)
        stepped[form] = (mine, b.stats(ids))
        for k in ids:
            b.download(k)
        b.close()
    for k, w in enumerate(worlds):
        P = _params(w, 1)
        probe, x64 = _fp64_system(w, P)
        ef = _errors(probe, P, x64, stepped["fast"][0][k])
        em = _errors(probe, P, x64, stepped["mixed"][0][k])
        sm = stepped["mixed"][1][k]
        print(f"\nbatched world {pick[k]} ({w.W}x{w.W} {w.config['workload']}): pressure fast {ef[0]:.2e} "
              f"mixed {em[0]:.2e}, velocity fast {ef[1]:.2e} mixed {em[1]:.2e} (of the velocity projected: fast "
              f"{ef[4]:.2e} mixed {em[4]:.2e}); mixed {sm.cycles} iterations")
        assert sm.rel_residual <= 1e-6
        assert sm.particles == stepped["fast"][1][k].particles
        assert em[0] <= 2 * ef[0] + 1e-5, (pick[k], ef[0], em[0])
        assert em[4] <= 2 * ef[4] + 1e-5, (pick[k], ef[4], em[4])
