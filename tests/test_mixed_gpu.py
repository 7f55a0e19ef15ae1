"""The mixed-precision form: coarse levels in binary16, FP32 CG vectors,
FP64 dots, norms and true-residual checks.  It is not bit-exact with the
FP32 forms; it must stop at a true relative residual of at most 1e-6 and
its pressure must agree with an FP64 solve of the same system as closely
as the FP32 form's does (relative L2 1e-4, the bar the oracle's FP32 solve
meets), and a world's mixed step must be the same alone and in a batch."""
import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import compare_worlds, params

pytestmark = pytest.mark.gpu

TOL = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
MIXED = TOL | abi.STEP_MIXED
PRE = ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER", "SEAL_JOIN", "SEAL_ANCHOR",
       "CLASSIFY", "SET_FACES", "UNPRESS", "DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR")


def _fp64_pressure(world, P):
    from oracle.oracle import Oracle
    probe = world.copy()
    o = Oracle(probe, W.element_table())
    for name in PRE:
        o.pass_(P, name)
    x64, _, rel = o.solve_f64(P, rel_tol=1e-12)
    assert rel <= 1e-12
    return x64


def _step(world, P, flags):
    from worldinagrain_b200 import fluid
    w = world.copy()
    h = fluid.LiquidStep(w, W.element_table())
    h.step(P, max_cycles=64, flags=flags | abi.STEP_SHIFTED_SET, tolerance=1e-6)
    st = h.stats()
    h.download()
    h.close()
    return w, st


@pytest.mark.parametrize("builder", [lambda: W.dam_break(256, 256, seed=1), lambda: W.disks_world(256, 256, n_disks=20, seed=4)])
def test_mixed_pressure_against_fp64_solve(builder):
    from worldinagrain_b200 import fluid
    world = builder()
    g = fluid.LiquidStep(world, W.element_table())
    for s in range(1, 4):
        g.step(params(world, s), max_cycles=64, flags=TOL, tolerance=1e-6)
    g.download()
    g.close()
    P = params(world, 4)
    x64 = _fp64_pressure(world, P)
    w32, st32 = _step(world, P, TOL)
    wm, stm = _step(world, P, MIXED)
    fluid_ = w32.field_cells()[:, 0, 2] > 0
    ref = x64[fluid_]
    e32 = np.linalg.norm(w32.field_cells()[:, 0, 0][fluid_] - ref) / np.linalg.norm(ref)
    em = np.linalg.norm(wm.field_cells()[:, 0, 0][fluid_] - ref) / np.linalg.norm(ref)
    assert stm.rel_residual <= 1e-6, stm.rel_residual
    assert stm.cycles <= 64
    assert e32 < 1e-4 and em < 1e-4, (e32, em)


def test_mixed_form_rounds_a_two_density_operator():
    """Water beside a denser liquid: the coarse levels' averaged densities and
    their coefficients are not all exact in binary16 (with one density they
    are: 1, 0 or -1, and betas of 1), so the mixed form's pressure differs
    from the FP32 form's, and both agree with the FP64 solve."""
    from worldinagrain_b200 import fluid
    world = W.two_liquids(192, 160, seed=5)
    g = fluid.LiquidStep(world, W.element_table())
    for s in range(1, 4):
        g.step(params(world, s), max_cycles=64, flags=TOL, tolerance=1e-6)
    g.download()
    g.close()
    P = params(world, 4)
    x64 = _fp64_pressure(world, P)
    w32, st32 = _step(world, P, TOL)
    wm, stm = _step(world, P, MIXED)
    fluid_ = w32.field_cells()[:, 0, 2] > 0
    ref = x64[fluid_]
    p32, pm = w32.field_cells()[:, 0, 0][fluid_], wm.field_cells()[:, 0, 0][fluid_]
    assert not np.array_equal(p32, pm)
    e32 = np.linalg.norm(p32 - ref) / np.linalg.norm(ref)
    em = np.linalg.norm(pm - ref) / np.linalg.norm(ref)
    assert stm.rel_residual <= 1e-6, stm.rel_residual
    assert e32 < 1e-4 and em < 1e-4, (e32, em)


def test_mixed_steps_keep_converging():
    from worldinagrain_b200 import fluid
    world = W.small_world(96, 80, seed=5, kind="moving")
    g = fluid.LiquidStep(world, W.element_table())
    n0 = None
    for s in range(1, 11):
        g.step(params(world, s), max_cycles=64, flags=MIXED, tolerance=1e-6)
        st = g.stats()
        assert st.rel_residual <= 1e-6, (s, st.rel_residual, st.cycles)
        n0 = n0 or st.particles
        assert st.particles == n0
    g.close()


def test_mixed_batch_matches_each_world_alone():
    from worldinagrain_b200 import fluid
    worlds = [W.dam_break(256, 256, seed=1), W.small_world(96, 80, seed=5, kind="obstacles"),
              W.small_world(48, 40, seed=2, kind="moving")]
    refs = []
    for w in worlds:
        r = w.copy()
        h = fluid.LiquidStep(r, W.element_table())
        # the mixed form's coarse kernel keeps its levels in FP32, the tile
        # kernels store theirs in 16 bits: alone, the world starts its coarse
        # kernel where the batch does (a batch's default, 4096 cells)
        h.set_launch("coarse_cells", 4096)
        for s in range(1, 4):
            h.step(params(r, s), max_cycles=64, flags=MIXED, tolerance=1e-6)
        h.download()
        h.close()
        refs.append(r)
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    for s in range(1, 4):
        b.step(range(3), [params(w, s) for w in mine], max_cycles=64, flags=MIXED, tolerance=1e-6)
    for k in range(3):
        b.download(k)
        d = compare_worlds(mine[k], refs[k], region_links=True)
        assert not d, f"world {k}: {d}"
    b.close()


def test_mixed_needs_tolerance_and_fp64_dots():
    from worldinagrain_b200 import fluid
    world = W.small_world(32, 32, seed=1, kind="dam")
    g = fluid.LiquidStep(world, W.element_table())
    with pytest.raises(fluid.WigError):
        g.step(params(world, 1), flags=abi.STEP_MIXED | abi.STEP_TOLERANCE, tolerance=1e-6)
    with pytest.raises(fluid.WigError):
        g.step(params(world, 1), flags=MIXED | abi.STEP_PLAIN, tolerance=1e-6)
    g.close()
