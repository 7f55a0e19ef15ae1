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
