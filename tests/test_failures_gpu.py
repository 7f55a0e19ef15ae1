"""The failure paths of the step on the GPU, each made on the host or by a
lowered bound: nothing here faults, traps or hangs the device, and each
case steps on normally afterwards.

- particles whose position or velocity is not finite (a NaN, an infinity,
  a position far outside the world): the step's clamps keep every index in
  the world (fluid.wgsl:3641-3644 bounds the advection's sub-steps, cellOf
  clamps positions, f32 -> i32 turns a NaN into 0), and the result is the
  oracle's, NaNs compared as NaNs;
- more particles than the buffers hold: those past the room are lost, the
  count says how many tried (fluid.wgsl:104-107, :827-830), and the stats
  read says WIG_E_CAPACITY;
- block bookkeeping the host corrupted (counts and lists past the world's
  blocks): sync and compact rebuild it before anything reads it;
- the union-find's retry bound and the persistent form's grid-barrier wait,
  lowered (wig_fluid_set_wait_limits) so they run out: the stats read says
  WIG_E_STATE, and a fresh step afterwards is the oracle's again;
- a tolerance-form solve cut short by max_cycles: WIG_E_NOT_CONVERGED, the
  report filled in all the same.
"""
import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import compare_worlds, params

pytestmark = pytest.mark.gpu

TOL = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
FORMS = {"plain": abi.STEP_PLAIN, "fast": 0}
SHIFTED = abi.STEP_SHIFTED_SET | abi.STEP_SHIFTED_FIRST


def _oracle(world):
    from oracle.oracle import Oracle
    return Oracle(world, W.element_table())


def _advanced(world, steps):
    o = _oracle(world)
    for s in range(1, steps + 1):
        o.step(params(world, s))
    return world


def _canonical_nans(world):
    """A copy whose f32 NaNs all have one bit pattern (a NaN's sign and
    payload are the hardware's choice, on the CPU and the GPU alike)."""
    out = world.copy()
    for name in ("sorted", "parts", "field", "cg"):
        f = getattr(out, name).view(np.float32)
        f[np.isnan(f)] = np.float32("nan")
    return out


def _poison(world):
    """Particles of `sorted` with non-finite positions and velocities, and
    positions far outside the world, spread over the liquid."""
    m = world.sorted[4:].reshape(3, world.cap, 4)[0].view(np.float32)
    a = world.sorted[4:].reshape(3, world.cap, 4)[2].view(np.float32)
    n = int(world.sorted[0])
    assert n > 64
    k = np.linspace(0, n - 1, 16).astype(int)
    inf, nan = np.float32("inf"), np.float32("nan")
    m[k[0:3], 2:4] = nan                 # velocity NaN
    m[k[3:6], 2] = inf                   # velocity +-inf
    m[k[3:6], 3] = -inf
    m[k[6:8], 0:2] = nan                 # position NaN
    m[k[8:10], 0] = inf                  # position at +inf
    m[k[10:12], 0:2] = np.float32(1e30)  # far outside the world
    m[k[12], 1] = -inf
    a[k[13:16]] = nan                    # affine velocity NaN


@pytest.mark.parametrize("form", ["plain", "fast"])
def test_non_finite_particles_step_without_fault_as_the_oracle(form):
    from worldinagrain_b200 import fluid
    world = _advanced(W.small_world(48, 40, seed=5, kind="obstacles"), 3)
    _poison(world)
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    got = world.copy()
    for s in range(4, 7):
        P = params(ref, s)
        so = o.step(P)
        g.step(P, flags=FORMS[form])
        st = g.stats()
        g.download(got)
        diffs = compare_worlds(_canonical_nans(got), _canonical_nans(ref), scratch=form != "plain")
        assert not diffs, f"step {s}: " + "; ".join(diffs)
        assert st.particles == so.particles
        assert np.all(np.isfinite(got.pressure()))
        F = got.L["face_count"]
        assert np.all(np.isfinite(got.field[8 * got.C: 8 * got.C + 4 * F]))
    g.close()


def test_capacity_overflow_is_reported_and_steps_go_on():
    """A 64 x 64 dam break seeds about 9,000 particles into room for 2,000:
    `parts`' count says how many tried (the oracle's too), the sorted
    buffer holds the room's worth, the stats read says WIG_E_CAPACITY, and
    the next steps run (reporting the overflow while it lasts)."""
    from worldinagrain_b200 import fluid
    base = W.dam_break(64, 64)
    world = W.World(64, 64, capacity=2000)
    world.cells[...] = base.cells
    world.config = base.config
    ref = world.copy()
    g = fluid.LiquidStep(world, W.element_table())
    _oracle(ref).step(params(ref, 1))
    got = world.copy()
    for s in range(1, 4):
        g.step(params(world, s))
        if s == 1:
            with pytest.raises(fluid.WigError, match="WIG_E_CAPACITY"):
                g.stats()
        else:
            try:
                g.stats()
            except fluid.WigError as e:
                assert "WIG_E_CAPACITY" in str(e)
        g.download(got)
        if s == 1:
            assert int(got.parts[0]) == int(ref.parts[0]) > got.cap
            assert int(got.sorted[0]) == int(ref.sorted[0]) == got.cap
        n = min(int(got.sorted[0]), got.cap)
        m = got.sorted[4:].reshape(3, got.cap, 4)[0].view(np.float32)[:n]
        assert np.all(np.isfinite(m[:, :2]))
        assert np.all((m[:, 0] >= 0) & (m[:, 0] <= got.W) & (m[:, 1] >= 0) & (m[:, 1] <= got.H))
    g.close()


def _mask_lists(world):
    """The blocks buffer with the list slots past their counts zeroed:
    compact writes each list's first `count` entries and leaves the rest."""
    B = world.L["block_count"]
    b = world.blocks.copy()
    na, nr = int(b[4 * B + abi.COUNT_ACTIVE]), int(b[4 * B + abi.COUNT_RETIRED])
    b[2 * B + na: 3 * B] = 0
    b[3 * B + nr: 4 * B] = 0
    b[4 * B + 9 + na:] = 0
    return b


@pytest.mark.parametrize("form", ["plain", "fast"])
def test_corrupted_block_bookkeeping_is_rebuilt(form):
    from worldinagrain_b200 import fluid
    world = _advanced(W.small_world(48, 40, seed=2, kind="obstacles"), 3)
    ref = world.copy()
    B = world.L["block_count"]
    bad = world.copy()
    bad.blocks[2 * B: 4 * B] = 0xFFFFFFFF                      # active and retired lists
    bad.blocks[4 * B + abi.COUNT_ACTIVE] = 0xFFFFFFFF          # counts past the blocks
    bad.blocks[4 * B + abi.COUNT_RETIRED] = 0xFFFFFFFF
    bad.blocks[4 * B + 9:] = 0xFFFFFFF0                        # per-block totals
    g = fluid.LiquidStep(bad, W.element_table())
    P = params(ref, 4)
    _oracle(ref).step(P)
    g.step(P, flags=FORMS[form])
    g.stats()
    g.download(bad)
    diffs = compare_worlds(bad, ref, grid=("cells", "counters", "field", "cg"), scratch=form != "plain")
    assert not diffs, "; ".join(diffs)
    assert np.array_equal(_mask_lists(bad), _mask_lists(ref))
    g.close()


@pytest.fixture
def lowered_limits():
    from worldinagrain_b200 import fluid
    yield fluid.set_wait_limits
    fluid.set_wait_limits(0, 0)


@pytest.mark.parametrize("form", ["plain", "fast"])
def test_union_find_bound_runs_out_and_reports(form, lowered_limits):
    from worldinagrain_b200 import fluid
    world = W.dam_break(64, 64)
    g = fluid.LiquidStep(world.copy(), W.element_table())
    lowered_limits(1, 0)
    g.step(params(world, 1), flags=FORMS[form])
    with pytest.raises(fluid.WigError, match="WIG_E_STATE.*union-find"):
        g.stats()
    lowered_limits(0, 0)
    # the device is fine: the same world from the start is the oracle's step
    # (the tiling parity set, as the handle has stepped once already)
    g.upload(world)
    ref = world.copy()
    _oracle(ref).step(params(ref, 1), flags=SHIFTED)
    g.step(params(world, 1), flags=FORMS[form] | SHIFTED)
    g.stats()
    got = g.download(world.copy())
    diffs = compare_worlds(got, ref, scratch=form != "plain")
    assert not diffs, "; ".join(diffs)
    g.close()


def test_persistent_grid_barrier_runs_out_and_reports(lowered_limits):
    from worldinagrain_b200 import fluid
    world = W.dam_break(128, 128)
    g = fluid.LiquidStep(world.copy(), W.element_table())
    lowered_limits(0, 1)
    g.step(params(world, 1), max_cycles=32, flags=TOL | abi.STEP_PERSISTENT, tolerance=1e-6)
    with pytest.raises(fluid.WigError, match="WIG_E_STATE.*barrier"):
        g.stats()
    lowered_limits(0, 0)
    g.upload(world)
    ref = world.copy()
    so = _oracle(ref).step(params(ref, 1), max_cycles=32, flags=TOL | SHIFTED, tolerance=1e-6)
    g.step(params(world, 1), max_cycles=32, flags=TOL | SHIFTED | abi.STEP_PERSISTENT, tolerance=1e-6)
    st = g.stats()
    assert st.cycles == so.cycles
    got = g.download(world.copy())
    diffs = compare_worlds(got, ref, scratch=True)
    assert not diffs, "; ".join(diffs)
    g.close()


def test_wait_limits_may_only_be_lowered():
    from worldinagrain_b200 import fluid
    with pytest.raises(fluid.WigError, match="WIG_E_ARG"):
        fluid.set_wait_limits(1 << 30, 0)
    fluid.set_wait_limits(0, 0)


@pytest.mark.parametrize("form", ["plain", "fast", "mixed"])
def test_solve_cut_short_reports_not_converged(form):
    """Two iterations cannot take the 256 x 256 dam break to 1e-6: the stats
    read says WIG_E_NOT_CONVERGED, its report filled in (two iterations, the
    residual above the tolerance); with enough iterations the same step is
    converged and reads clean."""
    from worldinagrain_b200 import fluid
    extra = {"plain": abi.STEP_PLAIN, "fast": 0, "mixed": abi.STEP_MIXED}[form]
    world = W.dam_break(256, 256)
    g = fluid.LiquidStep(world.copy(), W.element_table())
    g.step(params(world, 1), max_cycles=2, flags=TOL | extra | SHIFTED, tolerance=1e-6)
    with pytest.raises(fluid.NotConverged) as e:
        g.stats()
    st = e.value.stats
    assert st.cycles == 2 and st.rel_residual > 1e-6 and st.particles > 0
    assert g.stats(unconverged_ok=True).cycles == 2
    g.upload(world)
    g.step(params(world, 1), max_cycles=64, flags=TOL | extra | SHIFTED, tolerance=1e-6)
    st = g.stats()
    assert st.rel_residual <= 1e-6 and st.cycles > 2
    g.close()
