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


def test_snapshots_step_on_in_a_batch():
    """Snapshots of uneven worlds saved at different tiling parities, one of
    them of another particle layout, load into one batch and step on
    together, each world with its own saved parity, as the oracle steps each
    loaded world."""
    from oracle.oracle import Oracle
    from worldinagrain_b200 import abi, fluid
    tol = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
    made = [(48, 40, 4, 2), (96, 72, 6, 3), (64, 56, 8, 2)]
    refs, mine, nexts = [], [], []
    for k, (wd, ht, seed, steps) in enumerate(made):
        w = W.small_world(wd, ht, seed=seed, kind="obstacles")
        a = Oracle(w, W.element_table())
        for s in range(1, steps + 1):
            a.step(params(w, s), max_cycles=64, flags=tol, tolerance=1e-6)
        header, parts = snapshot.read(snapshot.save(w, state={"frameNo": steps, "shiftedFirst": bool(a.shifted.value)}))
        if k == 2:
            parts["particles0"] = parts["particles0"][:-48]
            parts["particles1"] = parts["particles1"][:-48]
        ref = snapshot.world_from(header, parts)
        Oracle(ref, W.element_table()).step(params(ref, steps + 1), max_cycles=64, flags=tol | snapshot.step_flags(ref),
                                            tolerance=1e-6)
        refs.append(ref)
        mine.append(snapshot.world_from(header, parts))
        nexts.append(steps + 1)
    assert mine[2].snapshot_migrated
    assert len({snapshot.step_flags(w) for w in mine}) == 2
    b = fluid.Batch(mine, W.element_table())
    ids = list(range(len(mine)))
    b.step(ids, [params(w, n) for w, n in zip(mine, nexts)], world_flags=[snapshot.step_flags(w) for w in mine],
           max_cycles=64, flags=tol, tolerance=1e-6)
    for k in ids:
        b.download(k)
        d = compare_worlds(mine[k], refs[k], region_links=True, scratch=True)
        assert not d, f"world {k}: {d}"
    b.close()


@pytest.mark.parametrize("pooled", [False, True])
def test_snapshots_served_step_on(pooled):
    """Snapshots served: each world's state goes up whole at its first
    admission (under a budget that forces evictions), its frames count on
    from the saved one, its first step takes its saved tiling parity, and
    after two requests each it holds what the oracle leaves."""
    from oracle.oracle import Oracle
    from worldinagrain_b200 import abi, fluid, serve
    tol = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
    made = [(48, 40, 4, 2), (96, 72, 6, 3), (64, 56, 8, 2), (40, 40, 2, 1)]
    refs, mine = [], []
    for k, (wd, ht, seed, steps) in enumerate(made):
        w = W.small_world(wd, ht, seed=seed, kind="obstacles")
        a = Oracle(w, W.element_table())
        for s in range(1, steps + 1):
            a.step(W.make_params(w, frame=s, seed=0x5eed, earth_g=w.config["earth_g"]), max_cycles=64, flags=tol,
                   tolerance=1e-6)
        header, parts = snapshot.read(snapshot.save(w, state={"frameNo": steps, "shiftedFirst": bool(a.shifted.value)}))
        if k == 2:
            parts["particles0"] = parts["particles0"][:-48]
            parts["particles1"] = parts["particles1"][:-48]
        ref = snapshot.world_from(header, parts)
        o = Oracle(ref, W.element_table())
        for n in (1, 2):
            P = W.make_params(ref, frame=steps + n, seed=0x5eed, earth_g=ref.config["earth_g"])
            o.step(P, max_cycles=64, flags=tol | (snapshot.step_flags(ref) if n == 1 else 0), tolerance=1e-6)
        refs.append(ref)
        mine.append(snapshot.world_from(header, parts))
    sizes = [fluid.world_bytes(w.W, w.H, w.L["liquid_per_cell"], w.cap) for w in mine]
    be = serve.GpuBackend(mine, W.element_table(), tol, 64, 1e-6, pool_bytes=3 * max(sizes) if pooled else None)
    srv = serve.Server(be, len(mine), sum(sorted(be.bytes)[-2:]))  # two worlds at a time
    srv.preload()
    arr = [(0.0, k) for k in (0, 1, 2, 3, 3, 2, 1, 0)]
    assert len(srv.run(arr)) == len(arr)
    assert srv.swaps_in > 0
    for k in list(srv.resident):
        be.fetch(k)
    grid = ("cells", "counters", "field", "blocks") if pooled else ("cells", "counters", "field", "blocks", "cg")
    for k, w in enumerate(mine):
        if pooled:
            # a pooled world keeps its field up to its coarse levels
            n = 4 * (2 * w.C + w.L["face_count"] + 2 * ((w.L["face_count"] + 3) // 4))
            w.field[n:] = refs[k].field[n:]
        d = compare_worlds(w, refs[k], grid=grid, particles=("sorted",), region_links=True, scratch=True)
        assert not d, f"world {k}: {d}"
    be.close()
