"""A world loaded from a snapshot into the GPU handle steps on as the world
it was saved from (the oracle stepping it throughout): the snapshot's
buffers and tiling parity are all the step needs."""
import pytest

from worldinagrain_b200 import snapshot
from worldinagrain_b200 import world as W

from .common import compare_worlds, params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("size", [(48, 40), (200, 136)])
def test_snapshot_loaded_on_the_gpu_steps_on(size):
    from oracle.oracle import Oracle
    from worldinagrain_b200 import fluid
    base = W.small_world(*size, seed=4, kind="obstacles")
    full = base.copy()
    o = Oracle(full, W.element_table())
    for s in range(1, 4):
        o.step(params(full, s))
    part = base.copy()
    a = Oracle(part, W.element_table())
    for s in range(1, 3):
        a.step(params(part, s))
    loaded = snapshot.load(snapshot.save(part, state={"frameNo": 2, "shiftedFirst": bool(a.shifted.value)}))
    g = fluid.LiquidStep(loaded, W.element_table())
    g.step(params(loaded, 3), flags=snapshot.step_flags(loaded))
    g.download()
    g.close()
    d = compare_worlds(loaded, full, region_links=True, scratch=True)
    assert not d, "; ".join(d)


def test_snapshot_of_another_particle_layout_reseeds_on_the_gpu():
    """A snapshot whose particles are laid out otherwise loads with none
    (migrateLiquid); its first GPU step seeds the liquid afresh as the
    oracle's does."""
    from oracle.oracle import Oracle
    from worldinagrain_b200 import fluid
    w = W.small_world(96, 72, seed=6, kind="obstacles")
    a = Oracle(w, W.element_table())
    for s in range(1, 3):
        a.step(params(w, s))
    header, parts = snapshot.read(snapshot.save(w, state={"frameNo": 2, "shiftedFirst": bool(a.shifted.value)}))
    parts["particles0"] = parts["particles0"][:-48]
    parts["particles1"] = parts["particles1"][:-48]
    ref = snapshot.world_from(header, parts)
    got = snapshot.world_from(header, parts)
    assert got.snapshot_migrated
    Oracle(ref, W.element_table()).step(params(ref, 3), flags=snapshot.step_flags(ref))
    g = fluid.LiquidStep(got, W.element_table())
    g.step(params(got, 3), flags=snapshot.step_flags(got))
    g.download()
    g.close()
    assert ref.sorted[0] > 0
    d = compare_worlds(got, ref, region_links=True, scratch=True)
    assert not d, "; ".join(d)
