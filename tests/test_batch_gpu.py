"""A batch of worlds stepped together through wig_batch_step: each world
leaves the same buffers as stepped alone (wig_fluid_step, the fast form)
and as the oracle, whichever worlds step beside it, on either lane, with
two lanes' steps in flight at once."""
import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import compare_worlds, params

pytestmark = pytest.mark.gpu

TOL = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS


def _mix():
    """Worlds of uneven sizes and kinds; the last one viscous."""
    return [
        W.small_world(32, 32, seed=7, kind="dam"),
        W.small_world(48, 40, seed=5, kind="obstacles"),
        W.small_world(40, 32, seed=3, kind="moving"),
        W.dam_break(64, 64, seed=1),
        W.small_world(72, 24, seed=9, kind="obstacles"),
        W.two_liquids(40, 32, seed=5),
    ]


def _flags_of(worlds):
    return [abi.STEP_VISCOUS if w.config["workload"] == "two_liquids" else 0 for w in worlds]


def _alone(world, steps, wflags, flags, seed_off=0):
    from worldinagrain_b200 import fluid
    w = world.copy()
    h = fluid.LiquidStep(w, W.element_table())
    for s in range(1, steps + 1):
        h.step(params(w, s + seed_off), max_cycles=64, flags=flags | wflags, tolerance=1e-6)
    h.download()
    st = h.stats()
    h.close()
    return w, st


def _same(a, b):
    return compare_worlds(a, b, region_links=True)


@pytest.mark.parametrize("flags", [0, TOL])
def test_batch_matches_each_world_alone(flags):
    from worldinagrain_b200 import fluid
    worlds = _mix()
    wf = _flags_of(worlds)
    ref = [_alone(w, 4, f, flags) for w, f in zip(worlds, wf)]
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    ids = list(range(len(mine)))
    for s in range(1, 5):
        b.step(ids, [params(w, s) for w in mine], world_flags=wf, max_cycles=64, flags=flags, tolerance=1e-6)
    st = b.stats(ids)
    for k, w in enumerate(mine):
        b.download(k)
        d = _same(w, ref[k][0])
        assert not d, f"world {k}: {d}"
        assert st[k].cycles == ref[k][1].cycles
        assert list(st[k].count) == list(ref[k][1].count)
    b.close()


def test_batch_matches_oracle():
    from oracle.oracle import Oracle
    from worldinagrain_b200 import fluid
    worlds = _mix()[:4]
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    ids = [0, 1, 2, 3]
    for s in range(1, 4):
        b.step(ids, [params(w, s) for w in mine], max_cycles=64, flags=TOL, tolerance=1e-6)
    for k, w in enumerate(worlds):
        o = Oracle(w.copy(), W.element_table())
        for s in range(1, 4):
            o.step(params(o.world, s), max_cycles=64, flags=TOL, tolerance=1e-6)
        b.download(k)
        d = compare_worlds(mine[k], o.world, region_links=True, scratch=True)
        assert not d, f"world {k}: {d}"
    b.close()


def test_subset_steps_leave_the_others_alone():
    from worldinagrain_b200 import fluid
    worlds = _mix()
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    wf = _flags_of(worlds)
    before = {k: mine[k].copy() for k in (1, 3, 4)}
    picked = [5, 0, 2]  # any order
    for s in range(1, 4):
        b.step(picked, [params(mine[k], s) for k in picked], world_flags=[wf[k] for k in picked], max_cycles=64,
               flags=TOL, tolerance=1e-6)
    for k in (1, 3, 4):
        b.download(k)
        assert not compare_worlds(mine[k], before[k]), k
    for k in picked:
        b.download(k)
        ref, _ = _alone(worlds[k], 3, wf[k], TOL)
        d = _same(mine[k], ref)
        assert not d, f"world {k}: {d}"
    b.close()


def test_two_lanes_in_flight_at_once():
    import torch
    from worldinagrain_b200 import fluid
    worlds = _mix()
    wf = _flags_of(worlds)
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    a_ids, b_ids = [0, 2, 4], [1, 3, 5]
    for s in range(1, 4):
        b.step(a_ids, [params(mine[k], s) for k in a_ids], world_flags=[wf[k] for k in a_ids], max_cycles=64,
               flags=TOL, tolerance=1e-6, lane=0, stream=s1.cuda_stream)
        b.step(b_ids, [params(mine[k], s) for k in b_ids], world_flags=[wf[k] for k in b_ids], max_cycles=64,
               flags=TOL, tolerance=1e-6, lane=1, stream=s2.cuda_stream)
    torch.cuda.synchronize()
    for k in range(len(mine)):
        b.download(k)
        ref, _ = _alone(worlds[k], 3, wf[k], TOL)
        d = _same(mine[k], ref)
        assert not d, f"world {k}: {d}"
    b.close()


def test_bookkeeping_only_world_in_a_batch():
    """A world whose step is bookkeeping only beside full ones: the same as
    its bookkeeping-only step alone."""
    from worldinagrain_b200 import fluid
    worlds = _mix()[:3]
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    wf = [0, abi.STEP_BOOKKEEPING_ONLY, 0]
    b.step([0, 1, 2], [params(w, 1) for w in mine], world_flags=wf, max_cycles=64, flags=TOL, tolerance=1e-6)
    for k in range(3):
        b.download(k)
        ref, _ = _alone(worlds[k], 1, wf[k], TOL)
        d = _same(mine[k], ref)
        assert not d, f"world {k}: {d}"
    b.close()


def test_batch_refuses_bad_lists():
    from worldinagrain_b200 import fluid
    mine = [w.copy() for w in _mix()[:2]]
    b = fluid.Batch(mine, W.element_table())
    P = [params(mine[0], 1)] * 2
    with pytest.raises(fluid.WigError):
        b.step([0, 0], P)
    with pytest.raises(fluid.WigError):
        b.step([0, 2], P)
    with pytest.raises(fluid.WigError):
        b.step([0], P[:1], lane=2)
    with pytest.raises(fluid.WigError):
        b.step([0], P[:1], flags=abi.STEP_PLAIN)
    b.close()


def test_batch_of_multi_level_worlds_matches_alone():
    """Worlds of the batched set whose levels go through the per-level
    tile kernels (sides 176 to 512: one to three levels above the coarse
    kernel's) beside one that has none: each the same as stepped alone,
    converged."""
    from worldinagrain_b200 import fluid
    picked = [2, 25, 9, 120, 135]  # sides 96, 176, 272, 400, 512
    worlds = W.multi_worlds(n=512, seed=2, only=picked)
    ref = [_alone(w, 3, 0, TOL) for w in worlds]
    mine = [w.copy() for w in worlds]
    b = fluid.Batch(mine, W.element_table())
    ids = list(range(len(mine)))
    for s in range(1, 4):
        b.step(ids, [params(w, s) for w in mine], max_cycles=64, flags=TOL, tolerance=1e-6)
    st = b.stats(ids)
    for k, w in enumerate(mine):
        b.download(k)
        d = _same(w, ref[k][0])
        assert not d, f"world {picked[k]}: {d}"
        assert st[k].cycles == ref[k][1].cycles
        assert st[k].rel_residual <= 1e-6, (picked[k], st[k].rel_residual)
    b.close()


def test_many_world_batch_is_deterministic():
    """96 worlds of the batched set (many tiles a CTA in each level kernel):
    two batches stepped alike leave the same buffers and stats, so no kernel
    reads a cell that another CTA of the same launch writes."""
    from worldinagrain_b200 import fluid
    picked = list(range(96))
    runs = []
    for _ in range(2):
        mine = W.multi_worlds(n=512, seed=2, only=picked)
        b = fluid.Batch(mine, W.element_table())
        ids = list(range(len(mine)))
        for s in range(1, 4):
            b.step(ids, [params(w, s) for w in mine], max_cycles=64, flags=TOL, tolerance=1e-6)
        st = b.stats(ids)
        for k in ids:
            b.download(k)
        b.close()
        runs.append((mine, [(x.cycles, x.rel_residual, tuple(x.count)) for x in st]))
    (wa, sa), (wb, sb) = runs
    for k in range(len(picked)):
        assert sa[k] == sb[k], (picked[k], sa[k], sb[k])
        assert sa[k][1] <= 1e-6, (picked[k], sa[k][1])
        d = _same(wa[k], wb[k])
        assert not d, f"world {picked[k]}: {d}"


def test_launch_shapes_change_no_result():
    """Every launch-shape knob at a value other than its default, the V-cycle
    handed to the coarse kernel at another depth: the same buffers and stats
    as the default shapes."""
    from worldinagrain_b200 import fluid
    picked = [2, 25, 9, 120]
    runs = []
    for shapes in ({}, {"coarse_cells": 512, "level_per_sm": 2, "cg_per_sm": 3, "relax_per_sm": 5}):
        mine = W.multi_worlds(n=512, seed=2, only=picked)
        b = fluid.Batch(mine, W.element_table())
        for k, v in shapes.items():
            b.set_launch(k, v)
        ids = list(range(len(mine)))
        for s in range(1, 4):
            b.step(ids, [params(w, s) for w in mine], max_cycles=64, flags=TOL, tolerance=1e-6)
        st = b.stats(ids)
        for k in ids:
            b.download(k)
        got = b.launch_shapes()
        b.close()
        runs.append((mine, [(x.cycles, x.rel_residual, tuple(x.count)) for x in st], got))
    (wa, sa, _), (wb, sb, gb) = runs
    assert gb == {"coarse_cells": 512, "level_per_sm": 2, "cg_per_sm": 3, "relax_per_sm": 5}
    for k in range(len(picked)):
        assert sa[k] == sb[k], (picked[k], sa[k], sb[k])
        d = _same(wa[k], wb[k])
        assert not d, f"world {picked[k]}: {d}"


def test_autotuned_batch_steps_as_the_untuned_one():
    """The tuner's profiled steps are the batch's steps: a tuned batch and
    one stepped alike with the default shapes end bit for bit the same."""
    from worldinagrain_b200 import fluid, tune
    picked = [2, 25, 9]
    n_steps = tune.steps_needed() + 2
    out = []
    for tuned in (False, True):
        mine = W.multi_worlds(n=512, seed=2, only=picked)
        b = fluid.Batch(mine, W.element_table())
        ids = list(range(len(mine)))
        s = [0]

        def prof_step():
            s[0] += 1
            return b.step_profile(ids, [params(w, s[0]) for w in mine], max_cycles=64, flags=TOL, tolerance=1e-6)

        if tuned:
            shapes, trials = tune.autotune(b, prof_step)
            assert set(trials) == {k for k, _, _ in tune.KNOBS}
        while s[0] < n_steps:
            prof_step()
        for k in ids:
            b.download(k)
        b.close()
        out.append(mine)
    for k in range(len(picked)):
        d = _same(out[0][k], out[1][k])
        assert not d, f"world {picked[k]}: {d}"
