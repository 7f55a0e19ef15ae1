"""A single world's coarse levels on a thread-block cluster: coarse_cells
above 4096 starts the coarse kernel at a level of up to 16384 cells, whose
levels of more than 1024 cells are cut into row strips over 8 CTAs' shared
memory (k_fCoarseCluster).

- the fast form bit for bit with the oracle, over worlds whose strips split
  evenly (dam 256x256 from its level 1, disks 512x512 and 1024x1024 from
  levels 2 and 3) and raggedly (a 300x200 dam: levels 150x100 down to 19x13,
  rows that 8 CTAs do not divide, odd widths);
- the mixed form, whose levels inside the coarse kernel stay FP32 where the
  tile kernels store them in 16 bits: converged, the same particles, and its
  pressure and velocity errors against an FP64 solve within the bound the
  mixed form is held to (twice the FP32 form's plus 1e-5);
- a batch of several worlds refuses the knob's cluster range."""
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .test_configs_gpu import _errors, _flags_of, _fp64_system, _oracle, _params, _same_step

pytestmark = pytest.mark.gpu

CLUSTER_CELLS = 16384

WORLDS = {
    "dam256": lambda: W.dam_break(256, 256, seed=2),
    "disks512": lambda: W.disks_world(512, 512, n_disks=60, seed=2),
    "disks1024": lambda: W.disks_world(1024, 1024, seed=2),
    "dam300x200": lambda: W.dam_break(300, 200, seed=2),
}


@pytest.mark.parametrize("name", list(WORLDS))
def test_cluster_coarse_levels_match_oracle(name):
    from worldinagrain_b200 import fluid
    world = WORLDS[name]()
    ref = world.copy()
    o = _oracle(ref)
    g = fluid.LiquidStep(world, W.element_table())
    g.set_launch("coarse_cells", CLUSTER_CELLS)
    assert g.get_launch("coarse_cells") == CLUSTER_CELLS
    got = world.copy()
    for s in range(1, 4):
        P = _params(ref, s)
        so = o.step(P, max_cycles=64, flags=_flags_of(s), tolerance=1e-6)
        g.step(P, max_cycles=64, flags=_flags_of(s), tolerance=1e-6)
        sg = g.stats()
        g.download(got)
        try:
            _same_step(got, ref, sg, so, scratch=True)
        except AssertionError as e:
            raise AssertionError(f"{name}, step {s}: {e}") from None
    g.close()


def test_cluster_coarse_levels_mixed_form_against_fp64_solve():
    from worldinagrain_b200 import fluid
    world = W.dam_break(256, 256, seed=2)
    P = _params(world, 1)
    out = {}
    for form, extra, cells in (("fast", 0, 4096), ("mixed", abi.STEP_MIXED, CLUSTER_CELLS)):
        w = world.copy()
        g = fluid.LiquidStep(w, W.element_table())
        g.set_launch("coarse_cells", cells)
        g.step(P, max_cycles=64, flags=_flags_of(1) | extra, tolerance=1e-6)
        out[form] = (w, g.stats())
        g.download()
        g.close()
    sm = out["mixed"][1]
    assert sm.rel_residual <= 1e-6
    assert sm.particles == out["fast"][1].particles
    probe, x64 = _fp64_system(world, P)
    ef = _errors(probe, P, x64, out["fast"][0])
    em = _errors(probe, P, x64, out["mixed"][0])
    print(f"\ndam 256x256 on a cluster, mixed: pressure {em[0]:.2e} (fast {ef[0]:.2e}), velocity of the projected "
          f"{em[4]:.2e} (fast {ef[4]:.2e}); {sm.cycles} iterations")
    assert em[0] <= 2 * ef[0] + 1e-5
    assert em[4] <= 2 * ef[4] + 1e-5


def test_batch_of_several_worlds_refuses_the_cluster_range():
    from worldinagrain_b200 import fluid
    worlds = [W.dam_break(64, 64, seed=2), W.dam_break(96, 64, seed=3)]
    b = fluid.Batch(worlds, W.element_table())
    with pytest.raises(fluid.WigError):
        b.set_launch("coarse_cells", CLUSTER_CELLS)
    assert b.get_launch("coarse_cells") == 4096
    b.set_launch("coarse_cells", 4096)
    b.close()
