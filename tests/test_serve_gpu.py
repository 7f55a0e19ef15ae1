"""The serving loop on the GPU: worlds admitted and evicted under a small
memory budget, steps batched over two lanes (with and without lane
pools), and every world's state after its requests the same, bit for bit,
as stepping it alone as many times."""
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W
from worldinagrain_b200 import serve

from .common import compare_worlds

pytestmark = pytest.mark.gpu

FLAGS = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS


def _worlds():
    out = [W.small_world(32 + 8 * (k % 4), 32, seed=k + 1, kind=("dam", "obstacles", "moving")[k % 3])
           for k in range(8)]
    out.append(W.dam_break(64, 64, seed=2))
    return out


def _alone(world, n_steps):
    from worldinagrain_b200 import fluid
    w = world.copy()
    h = fluid.LiquidStep(w, W.element_table())
    for s in range(1, n_steps + 1):
        P = W.make_params(w, frame=s, seed=0x5eed, earth_g=w.config["earth_g"])
        h.step(P, max_cycles=64, flags=FLAGS, tolerance=1e-6)
    h.download()
    h.close()
    return w


@pytest.mark.parametrize("pooled", [False, True])
def test_served_worlds_match_stepping_alone(pooled):
    from worldinagrain_b200 import fluid
    base = _worlds()
    mine = [w.copy() for w in base]
    sizes = [fluid.world_bytes(w.W, w.H, w.L["liquid_per_cell"], w.cap) for w in mine]
    be = serve.GpuBackend(mine, W.element_table(), FLAGS, 64, 1e-6, pool_bytes=3 * max(sizes) if pooled else None)
    # room for about half of the worlds: requests force evictions
    budget = sum(sorted(be.bytes)[-5:])
    srv = serve.Server(be, len(mine), budget)
    srv.preload()
    arr = serve.poisson_arrivals(rate=400.0, n_requests=60, n_worlds=len(mine), seed=7)
    done = srv.run(arr)
    assert len(done) == 60
    assert srv.swaps_in > 0
    counts = [0] * len(mine)
    for _, k in arr:
        counts[k] += 1
    for k in list(srv.resident):
        be.fetch(k)
    grid = ("cells", "counters", "field", "blocks") if pooled else ("cells", "counters", "field", "blocks", "cg")
    for k, w in enumerate(mine):
        ref = _alone(base[k], counts[k])
        if pooled:
            # a pooled world keeps its field up to its coarse levels
            n = 4 * (2 * w.C + w.L["face_count"] + 2 * ((w.L["face_count"] + 3) // 4))
            w.field[n:] = ref.field[n:]
        d = compare_worlds(w, ref, grid=grid, particles=("sorted",), region_links=True, scratch=True)
        assert not d, f"world {k} ({counts[k]} steps): {d}"
    be.close()


@pytest.mark.parametrize("pooled", [False, True])
def test_launch_shape_changes_between_served_steps(pooled):
    """Launch shapes changed twice between requests (the coarse kernel's depth
    among them, worlds with levels above it included): every world still
    ends as stepping it alone."""
    from worldinagrain_b200 import fluid
    base = _worlds()[:5] + [W.dam_break(256, 256, seed=3), W.dam_break(160, 128, seed=4)]
    mine = [w.copy() for w in base]
    sizes = [fluid.world_bytes(w.W, w.H, w.L["liquid_per_cell"], w.cap) for w in mine]
    be = serve.GpuBackend(mine, W.element_table(), FLAGS, 64, 1e-6, pool_bytes=3 * max(sizes) if pooled else None)
    srv = serve.Server(be, len(mine), sum(be.bytes))
    srv.preload()
    counts = [0] * len(mine)
    phases = ({"coarse_cells": 1024, "level_per_sm": 2, "cg_per_sm": 3, "relax_per_sm": 5},
              {"coarse_cells": 4096, "level_per_sm": 8, "cg_per_sm": 8, "relax_per_sm": 16}, None)
    for i, shapes in enumerate(phases):
        arr = serve.poisson_arrivals(rate=400.0, n_requests=20, n_worlds=len(mine), seed=11 + i)
        assert len(srv.run(arr)) == 20
        for _, k in arr:
            counts[k] += 1
        if shapes:
            for name, v in shapes.items():
                be.set_launch(name, v)
    for k in list(srv.resident):
        be.fetch(k)
    grid = ("cells", "counters", "field", "blocks") if pooled else ("cells", "counters", "field", "blocks", "cg")
    for k, w in enumerate(mine):
        ref = _alone(base[k], counts[k])
        if pooled:
            n = 4 * (2 * w.C + w.L["face_count"] + 2 * ((w.L["face_count"] + 3) // 4))
            w.field[n:] = ref.field[n:]
        d = compare_worlds(w, ref, grid=grid, particles=("sorted",), region_links=True, scratch=True)
        assert not d, f"world {k} ({counts[k]} steps): {d}"
    be.close()
