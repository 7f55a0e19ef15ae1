"""The serving loop's scheduling on the CPU, over a fake device: every
request served once, a world never in two steps at once, the memory
budget and the lane pools never exceeded, least-recently-used eviction,
both lanes used."""
import collections

import pytest

from worldinagrain_b200 import serve


class FakeBackend:
    """Steps finish after `step_s` of the fake clock; records everything."""

    def __init__(self, sizes, step_s, clock, step_sizes=None, pool=None):
        self.sizes = sizes
        self.step_sizes = step_sizes or [0] * len(sizes)
        self.pool = pool
        self.step_s = step_s
        self.clock = clock
        self.resident = set()
        self.log = []
        self.inflight = collections.Counter()

    def world_bytes(self, k):
        return self.sizes[k]

    def step_bytes(self, k):
        return self.step_sizes[k]

    def lane_capacity(self, lane):
        return self.pool

    def admit(self, k):
        assert k not in self.resident
        self.resident.add(k)
        self.log.append(("admit", k))

    def evict(self, k):
        assert k in self.resident and self.inflight[k] == 0
        self.resident.remove(k)
        self.log.append(("evict", k))

    def launch(self, lane, ids):
        for k in ids:
            assert k in self.resident
            assert self.inflight[k] == 0, "a world in two steps at once"
            self.inflight[k] += 1
        if self.pool is not None:
            assert sum(self.step_sizes[k] for k in ids) <= self.pool
        self.log.append(("step", lane, tuple(ids)))
        return [self.clock.t + self.step_s, ids]

    def done(self, token):
        if self.clock.t >= token[0]:
            for k in token[1]:
                self.inflight[k] -= 1
            token[1] = []
            return True
        return False


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-4  # every look at the clock moves it on
        return self.t


@pytest.mark.parametrize("budget", [10_000, 450])
def test_every_request_served_once_within_budget(budget):
    clock = FakeClock()
    sizes = [50 + 10 * (k % 7) for k in range(20)]
    be = FakeBackend(sizes, step_s=0.003, clock=clock)
    srv = serve.Server(be, len(sizes), budget, clock=clock)
    srv.preload()
    arr = serve.poisson_arrivals(rate=2000.0, n_requests=300, n_worlds=len(sizes), seed=3)
    done = srv.run(arr)
    assert sorted(r.rid for r in done) == list(range(300))
    assert all(r.t_done >= r.t_start >= r.t_arrival for r in done)
    used = 0
    for ev in be.log:
        if ev[0] == "admit":
            used += sizes[ev[1]]
            assert used <= budget
        elif ev[0] == "evict":
            used -= sizes[ev[1]]
    assert {ev[1] for ev in be.log if ev[0] == "step"} == {0, 1}
    if budget < sum(sizes):
        assert srv.swaps_out > 0 and srv.swaps_in > 0


def test_lane_pool_bounds_each_step():
    clock = FakeClock()
    be = FakeBackend([10] * 12, step_s=0.002, clock=clock, step_sizes=[3 + k % 4 for k in range(12)], pool=12)
    srv = serve.Server(be, 12, 10_000, clock=clock)
    srv.preload()
    done = srv.run(serve.poisson_arrivals(5000.0, 200, 12, seed=4))
    assert len(done) == 200
    steps = [ev for ev in be.log if ev[0] == "step"]
    assert max(len(ev[2]) for ev in steps) > 1


def test_requests_of_one_world_run_in_order():
    clock = FakeClock()
    be = FakeBackend([10] * 3, step_s=0.002, clock=clock)
    srv = serve.Server(be, 3, 1000, clock=clock)
    srv.preload()
    done = sorted(srv.run([(0.0001 * i, 1) for i in range(10)]), key=lambda r: r.rid)
    for a, b in zip(done, done[1:]):
        assert b.t_start >= a.t_done


def test_one_at_a_time_baseline_steps_single_worlds():
    clock = FakeClock()
    be = FakeBackend([10] * 5, step_s=0.001, clock=clock)
    srv = serve.Server(be, 5, 1000, one_at_a_time=True, clock=clock)
    srv.preload()
    done = srv.run(serve.poisson_arrivals(1000.0, 50, 5, seed=1))
    assert len(done) == 50
    assert all(len(ev[2]) == 1 and ev[1] == 0 for ev in be.log if ev[0] == "step")


def test_eviction_is_least_recently_used():
    clock = FakeClock()
    be = FakeBackend([100] * 4, step_s=0.001, clock=clock)
    srv = serve.Server(be, 4, 300, clock=clock)
    srv.preload()  # worlds 0, 1, 2
    assert list(srv.resident) == [0, 1, 2]
    srv.run([(0.0, 1), (0.01, 0), (0.02, 3)])
    assert [ev[1] for ev in be.log if ev[0] == "evict"] == [2]


def test_merge_parts_pools_latencies_and_sums_throughput():
    a = {"lat_ms": [1.0, 2.0, 3.0], "swapped": [False] * 3, "cells": 300, "t0": 0.0, "t1": 1.0}
    b = {"lat_ms": [10.0], "swapped": [True], "cells": 100, "t0": 0.5, "t1": 1.0}
    m = serve.merge_parts([a, b])
    assert m["requests"] == 4
    assert m["p50_ms"] == 2.5
    assert m["mcells_per_s"] == round((300 / 1.0 + 100 / 0.5) / 1e6, 3)
    assert m["swapped_requests"] == 1 and m["p50_ms_resident"] == 2.0


def test_snapshot_worlds_carry_their_state_into_the_backend():
    """The GPU backend's bookkeeping for worlds loaded from snapshots, without
    a device: such a world uploads whole at its first admission, its frames
    count on from the saved one, and only its first step carries the saved
    tiling parity."""
    from worldinagrain_b200 import abi, snapshot
    from worldinagrain_b200 import world as W
    fresh = W.small_world(32, 32, seed=1, kind="dam")
    loaded = snapshot.load(snapshot.save(W.small_world(48, 40, seed=2, kind="dam"),
                                         state={"frameNo": 7, "shiftedFirst": True}))
    be = serve.GpuBackend.__new__(serve.GpuBackend)  # the bookkeeping only, no device
    be.worlds = [fresh, loaded]
    be.seed = 1
    be._init_states(be.worlds)
    assert be.has_state == [False, True] and be.frames == [0, 7]
    # the saved parity: shiftedFirst True, flipped before the step's first relaxation
    assert be.first_flags == [0, abi.STEP_SHIFTED_SET]
    wf = be._world_flags([1, 0])
    assert list(wf) == [abi.STEP_SHIFTED_SET, 0]
    P = be._next_params([1, 0])
    assert [p.frame for p in P] == [8, 1]
    assert be.has_state == [True, True]
    assert be._world_flags([0, 1]) is None  # later steps: the handle flips the parity itself


def test_requests_that_can_never_fit_are_refused_not_left_pending():
    """A world larger than the whole budget, or whose step borrows more than
    a lane pool holds, can never be admitted: its requests are refused on
    arrival (the loop ends, the budget holds) and the rest are served."""
    clock = FakeClock()
    sizes = [50, 50, 5000, 50]
    be = FakeBackend(sizes, step_s=0.002, clock=clock, step_sizes=[3, 30, 3, 3], pool=12)
    srv = serve.Server(be, len(sizes), 1000, clock=clock)
    srv.preload()
    assert 2 not in srv.resident
    arr = [(0.0005 * i, i % 4) for i in range(40)]
    done = srv.run(arr)
    assert len(done) == 40
    refused = [r for r in done if r.refused]
    assert {r.world for r in refused} == {1, 2} and len(refused) == 20
    assert "budget" in next(r for r in refused if r.world == 2).refused
    assert "lane pool" in next(r for r in refused if r.world == 1).refused
    assert all(ev[0] != "admit" or ev[1] != 2 for ev in be.log)
    s = serve.latency_summary(done, lambda k: 1)
    assert s["requests"] == 20 and s["refused_requests"] == 20
    part = serve.latency_part(done, lambda k: 1)
    assert serve.merge_parts([part])["refused_requests"] == 20
