"""Serving many liquid worlds on one GPU: step requests arrive at any time
for any of the resident worlds; the server admits them as step lanes and
device memory free up and batches the pending ones of different sizes into
one batched step (wig_batch_step: each pass one launch over all the worlds
in the step), keeping every world's state on the device between its steps.

Continuous batching: the batch has two step lanes.  While one lane's step
runs, requests that arrive are admitted into the other lane's next step as
soon as it is free, so the two steps' work overlaps on the device; a world
is never in two steps at once (a second request for it waits for the
first).  Memory: worlds are admitted to the device (their memory allocated,
their state uploaded) under a byte budget; when a request needs a world that
is not resident, idle resident worlds are evicted least-recently-used first
(their state downloaded to the host).  With lane pools (GpuBackend
pool_bytes), a resident world holds only what persists between its steps,
and each step borrows the rest (its `parts` and `cg` buffers and the
solve's scratch) from its lane's pool, which bounds the worlds of one step.

The reference has no counterpart (its Simulation steps one world per
frame); a world's step here is the same step as stepping it alone.

The device operations sit behind a small backend interface (GpuBackend);
the scheduling logic runs unchanged over a fake one on the CPU in tests.
"""
import collections
import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi, snapshot


@dataclass
class Request:
    rid: int
    world: int
    t_arrival: float
    t_start: float = 0.0
    t_done: float = 0.0
    lane: int = -1
    swapped: bool = False
    refused: str = ""  # why the request was refused on arrival ("" if served)


@dataclass
class LaneState:
    busy: bool = False
    requests: list = field(default_factory=list)
    token: object = None
    t_launch: float = 0.0


class GpuBackend:
    """The device side: a deferred wig_batch over the worlds (host World
    objects hold the state of the worlds not resident), a CUDA stream a
    lane, and (pool_bytes) a pool a lane for the steps' borrowed memory."""

    def __init__(self, worlds, elems, flags, max_cycles, tolerance, pool_bytes=None, seed=0x5eed):
        import torch
        from . import fluid
        self.torch = torch
        self.fluid = fluid
        self.worlds = worlds
        self.flags = flags
        self.max_cycles = max_cycles
        self.tolerance = tolerance
        self.seed = seed
        L = fluid.lib()
        self._setup_funcs(L)
        descs = (abi.WorldDesc * len(worlds))(*[w.desc() for w in worlds])
        h = C.c_void_p()
        fluid.check(L.wig_batch_create_deferred(descs, len(worlds), elems, len(elems), C.byref(h)),
                    "wig_batch_create_deferred")
        self.h = h
        self.streams = [torch.cuda.Stream(), torch.cuda.Stream()]
        self._init_states(worlds)
        self.pooled = pool_bytes is not None
        self.pool = pool_bytes
        split = [self._split(w) for w in worlds]
        if self.pooled:
            for lane in range(2):
                fluid.check(L.wig_batch_set_lane_pool(self.h, lane, int(pool_bytes)), "wig_batch_set_lane_pool")
            self.bytes = [p for p, _ in split]
            self.step_bytes_ = [t for _, t in split]
        else:
            self.bytes = [p + t for p, t in split]
            self.step_bytes_ = [0] * len(worlds)
        self.names = [(which, name) for which, name in enumerate(abi.BUFFER_NAMES)
                      if not (self.pooled and name in ("parts", "cg"))]

    def _init_states(self, worlds):
        """Per world: whether it holds a state, its frame count, the flags of
        its first step. A world loaded from a snapshot (snapshot.load) holds
        one: all of its buffers go up at its first admission, its frames
        count on from the saved one, and its first step sets the saved
        tiling parity."""
        self.has_state = [hasattr(w, "snapshot_state") for w in worlds]
        self.frames = [int(w.snapshot_state.get("frameNo", 0)) if s else 0 for w, s in zip(worlds, self.has_state)]
        self.first_flags = [snapshot.step_flags(w) if s else 0 for w, s in zip(worlds, self.has_state)]

    @staticmethod
    def _setup_funcs(L):
        for name, args, res in (
                ("wig_batch_create_deferred", [C.POINTER(abi.WorldDesc), C.c_uint32, C.POINTER(abi.Elem), C.c_uint32,
                                               C.POINTER(C.c_void_p)], C.c_int),
                ("wig_batch_admit", [C.c_void_p, C.c_uint32, C.c_void_p], C.c_int),
                ("wig_batch_evict", [C.c_void_p, C.c_uint32, C.c_void_p], C.c_int),
                ("wig_batch_resident_bytes", [C.c_void_p], C.c_uint64),
                ("wig_batch_set_lane_pool", [C.c_void_p, C.c_uint32, C.c_uint64], C.c_int),
                ("wig_batch_world_bytes_split", [C.POINTER(abi.WorldDesc), C.POINTER(C.c_uint64),
                                                 C.POINTER(C.c_uint64)], C.c_int)):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res

    def _split(self, w):
        d = abi.WorldDesc(w.W, w.H, w.L["liquid_per_cell"], w.cap)
        p, t = C.c_uint64(), C.c_uint64()
        self.fluid.check(self.fluid.lib().wig_batch_world_bytes_split(C.byref(d), C.byref(p), C.byref(t)),
                         "wig_batch_world_bytes_split")
        return p.value, t.value

    def world_bytes(self, k):
        """Device bytes world k holds while resident."""
        return self.bytes[k]

    def step_bytes(self, k):
        """Bytes world k borrows from a lane's pool for a step (0: none)."""
        return self.step_bytes_[k]

    def lane_capacity(self, lane):
        return self.pool

    def admit(self, k):
        """Allocates world k on the device and uploads its host state (only
        its cells when it has never stepped and was not loaded from a
        snapshot: the rest is zero, as the new memory is)."""
        L = self.fluid.lib()
        s = C.c_void_p(self.streams[0].cuda_stream)
        self.fluid.check(L.wig_batch_admit(self.h, k, s), "wig_batch_admit")
        w = self.worlds[k]
        for which, name in (self.names if self.has_state[k] else [(0, "cells")]):
            arr = np.ascontiguousarray(getattr(w, name))
            self.fluid.check(L.wig_batch_upload(self.h, k, which, arr.ctypes.data, 0, arr.nbytes, s), "upload")

    def fetch(self, k):
        """Downloads resident world k's state to its host buffers."""
        L = self.fluid.lib()
        self.torch.cuda.synchronize()
        s = C.c_void_p(self.streams[0].cuda_stream)
        w = self.worlds[k]
        for which, name in self.names:
            arr = getattr(w, name)
            self.fluid.check(L.wig_batch_download(self.h, k, which, arr.ctypes.data, 0, arr.nbytes, s), "download")

    def evict(self, k):
        """Downloads world k's state to its host buffers and frees it."""
        self.fetch(k)
        self.fluid.check(self.fluid.lib().wig_batch_evict(self.h, k, C.c_void_p(self.streams[0].cuda_stream)),
                         "wig_batch_evict")

    def _next_params(self, ids):
        """The next step's Params of worlds `ids` (their frames advanced)."""
        P = (abi.Params * len(ids))()
        for i, k in enumerate(ids):
            self.frames[k] += 1
            self.has_state[k] = True
            w = self.worlds[k]
            p = P[i]
            p.size[0], p.size[1] = w.W, w.H
            p.frame = self.frames[k]
            p.seed = self.seed
            p.dx = 1.0
            p.earth_g = w.config["earth_g"]
            p.dt = 1.0 / 120.0
        return P

    def _world_flags(self, ids):
        """The per-world flags of the next step of worlds `ids` (the saved
        tiling parity of a snapshot's first step), or None when all are 0."""
        wf = [self.first_flags[k] for k in ids]
        for k in ids:
            self.first_flags[k] = 0
        return (C.c_uint32 * len(ids))(*wf) if any(wf) else None

    def launch(self, lane, ids):
        """One batched step of worlds `ids` on `lane`; returns a token."""
        n = len(ids)
        wf_a = self._world_flags(ids)
        P = self._next_params(ids)
        ids_a = (C.c_uint32 * n)(*ids)
        stream = self.streams[lane]
        self.fluid.check(self.fluid.lib().wig_batch_step(self.h, lane, ids_a, n, P, wf_a, self.max_cycles, self.flags,
                                                         self.tolerance, C.c_void_p(stream.cuda_stream)),
                         "wig_batch_step")
        ev = self.torch.cuda.Event()
        ev.record(stream)
        return ev

    def done(self, token):
        return token.query()

    # -- launch shapes (tune.autotune's interface)
    def get_launch(self, knob):
        v = C.c_uint32()
        self.fluid.check(self.fluid.lib().wig_batch_get_launch(self.h, abi.LAUNCH_KNOBS[knob], C.byref(v)),
                         "wig_batch_get_launch")
        return v.value

    def set_launch(self, knob, value):
        self.torch.cuda.synchronize()
        self.fluid.check(self.fluid.lib().wig_batch_set_launch(self.h, abi.LAUNCH_KNOBS[knob], int(value)),
                         "wig_batch_set_launch")

    def launch_shapes(self):
        return {name: self.get_launch(name) for name in abi.LAUNCH_KNOBS}

    def autotune(self, resident, lane=0):
        """Tunes the batch's launch shapes (tune.autotune) on profiled steps
        of resident worlds, as many as one lane's pool takes; those worlds
        step as they would in service. Returns the shapes and the trials."""
        from . import tune
        ids, used = [], 0
        for k in resident:
            b = self.step_bytes_[k]
            if self.pool is not None and used + b > self.pool:
                continue
            ids.append(k)
            used += b
        ms = (C.c_float * abi.PROFILE_SLOTS)()
        calls = (C.c_uint32 * abi.PROFILE_SLOTS)()
        ids_a = (C.c_uint32 * len(ids))(*ids)
        stream = self.streams[lane]

        def prof_step():
            wf_a = self._world_flags(ids)
            P = self._next_params(ids)
            self.fluid.check(self.fluid.lib().wig_batch_step_profile(
                self.h, lane, ids_a, len(ids), P, wf_a, self.max_cycles, self.flags, self.tolerance,
                C.c_void_p(stream.cuda_stream), ms, calls), "wig_batch_step_profile")
            return {abi.PROFILE_NAMES[k]: (ms[k], calls[k]) for k in range(abi.PROFILE_SLOTS) if calls[k]}

        return tune.autotune(self, prof_step)

    def stats(self, ids):
        """The worlds' last reports.  A world whose solve stopped short of the
        tolerance is reported (its rel_residual says so), not raised: one
        world's hard step does not stop the serving loop."""
        out = (abi.Stats * len(ids))()
        ids_a = (C.c_uint32 * len(ids))(*ids)
        rc = self.fluid.lib().wig_batch_read_stats(self.h, ids_a, len(ids), out)
        if rc != self.fluid.E_NOT_CONVERGED:
            self.fluid.check(rc, "wig_batch_read_stats")
        return list(out)

    def close(self):
        if self.h:
            self.torch.cuda.synchronize()
            self.fluid.lib().wig_batch_destroy(self.h)
            self.h = None


class Server:
    """The request loop over a backend: admission by memory budget, two
    lanes, continuous batching.  max_batch caps the worlds of one step
    (None: all that are ready and fit the lane); one_at_a_time steps a
    single world per launch on one lane (the one-world-at-a-time
    baseline)."""

    def __init__(self, backend, n_worlds, budget_bytes, max_batch=None, one_at_a_time=False, clock=time.perf_counter):
        self.be = backend
        self.n = n_worlds
        self.budget = budget_bytes
        self.max_batch = 1 if one_at_a_time else max_batch
        self.lanes = [LaneState()] if one_at_a_time else [LaneState(), LaneState()]
        self.clock = clock
        self.resident = collections.OrderedDict()  # world -> None, least recently used first
        self.resident_bytes = 0
        self.in_flight = set()
        self.swaps_in = 0
        self.swaps_out = 0

    # -- memory
    def preload(self, order=None):
        """Admits worlds in `order` (default 0..n-1) while they fit the budget."""
        for k in (order if order is not None else range(self.n)):
            b = self.be.world_bytes(k)
            if self.resident_bytes + b > self.budget:
                continue
            self.be.admit(k)
            self.resident[k] = None
            self.resident_bytes += b

    def _make_room(self, need, protect):
        """Evicts idle resident worlds, least recently used first, until
        `need` more bytes fit; False if that is not possible now."""
        if self.resident_bytes + need <= self.budget:
            return True
        victims, freed = [], 0
        for k in self.resident:
            if k in self.in_flight or k in protect:
                continue
            victims.append(k)
            freed += self.be.world_bytes(k)
            if self.resident_bytes - freed + need <= self.budget:
                break
        if self.resident_bytes - freed + need > self.budget:
            return False
        for k in victims:
            self.be.evict(k)
            del self.resident[k]
            self.resident_bytes -= self.be.world_bytes(k)
            self.swaps_out += 1
        return True

    def _ensure(self, k, protect):
        if k in self.resident:
            self.resident.move_to_end(k)
            return True, False
        need = self.be.world_bytes(k)
        if need > self.budget or not self._make_room(need, protect):
            return False, False
        self.be.admit(k)
        self.resident[k] = None
        self.resident_bytes += need
        self.swaps_in += 1
        return True, True

    def refusal(self, k):
        """Why a request for world k can never be served ("" if it can): its
        world's memory is above the whole budget, or its step's borrowed
        memory above a lane pool."""
        need = self.be.world_bytes(k)
        if need > self.budget:
            return f"world {k} needs {need} bytes resident, above the {self.budget}-byte budget"
        cap = self.be.lane_capacity(0)
        if cap is not None and self.be.step_bytes(k) > cap:
            return f"a step of world {k} borrows {self.be.step_bytes(k)} bytes, above a lane pool's {cap}"
        return ""

    # -- the loop
    def _complete(self, lane_id, now, finished):
        lane = self.lanes[lane_id]
        for r in lane.requests:
            r.t_done = now
            self.in_flight.discard(r.world)
            finished.append(r)
        lane.busy = False
        lane.requests = []
        lane.token = None

    def _launch(self, lane_id, pending, now):
        lane = self.lanes[lane_id]
        picked, worlds, rest = [], set(), collections.deque()
        cap = self.be.lane_capacity(lane_id)
        used = 0
        while pending:
            r = pending.popleft()
            if (r.world in self.in_flight or r.world in worlds
                    or (self.max_batch is not None and len(picked) >= self.max_batch)):
                rest.append(r)
                continue
            need = self.be.step_bytes(r.world) if cap is not None else 0
            if cap is not None and used + need > cap:
                rest.append(r)
                continue
            ok, swapped = self._ensure(r.world, worlds)
            if not ok:
                rest.append(r)
                continue
            r.swapped = swapped
            picked.append(r)
            worlds.add(r.world)
            used += need
        pending.extendleft(reversed(rest))
        if not picked:
            return False
        for r in picked:
            r.t_start = now
            r.lane = lane_id
            self.in_flight.add(r.world)
        lane.token = self.be.launch(lane_id, [r.world for r in picked])
        lane.requests = picked
        lane.busy = True
        lane.t_launch = now
        return True

    def run(self, arrivals):
        """Serves arrivals [(t_seconds, world)] (sorted by time, times from
        the start of the run); returns the finished Requests."""
        reqs = [Request(i, int(w), float(t)) for i, (t, w) in enumerate(arrivals)]
        pending = collections.deque()
        finished = []
        t0 = self.clock()
        i, total = 0, len(reqs)
        while len(finished) < total:
            now = self.clock() - t0
            while i < total and reqs[i].t_arrival <= now:
                # a request that no eviction can make room for is refused at
                # once, not left pending for ever
                why = self.refusal(reqs[i].world)
                if why:
                    reqs[i].refused = why
                    reqs[i].t_start = reqs[i].t_done = now
                    finished.append(reqs[i])
                else:
                    pending.append(reqs[i])
                i += 1
            for lane_id, lane in enumerate(self.lanes):
                if lane.busy and self.be.done(lane.token):
                    self._complete(lane_id, self.clock() - t0, finished)
            launched = False
            for lane_id, lane in enumerate(self.lanes):
                if not lane.busy and pending:
                    launched |= self._launch(lane_id, pending, self.clock() - t0)
            if not launched and not pending and i < total and not any(l.busy for l in self.lanes):
                wait = reqs[i].t_arrival - (self.clock() - t0)  # idle until the next arrival
                if wait > 0.0005:
                    time.sleep(wait - 0.0002)
        return finished


def poisson_arrivals(rate, n_requests, n_worlds, seed):
    """n_requests step requests at a Poisson total rate (per second), each
    for a world drawn uniformly; sorted (time, world) pairs."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    w = rng.integers(0, n_worlds, n_requests)
    return list(zip(t.tolist(), w.tolist()))


def latency_summary(finished, cells_of):
    """p50 / p99 / mean latency (ms, arrival to completion seen by the
    host), throughput (Mcells/s and steps/s over the run) and the requests
    that waited for their world to be swapped in, over the requests served
    (refused ones are counted apart)."""
    refused = sum(1 for r in finished if r.refused)
    finished = [r for r in finished if not r.refused]
    if not finished:
        return {"requests": 0, "refused_requests": refused}
    lat = np.array([r.t_done - r.t_arrival for r in finished]) * 1e3
    span = max(r.t_done for r in finished) - min(r.t_arrival for r in finished)
    cells = sum(cells_of(r.world) for r in finished)
    hit = np.array([not r.swapped for r in finished])
    out = {
        "requests": len(finished),
        "p50_ms": round(float(np.percentile(lat, 50)), 3),
        "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "mean_ms": round(float(lat.mean()), 3),
        "mcells_per_s": round(cells / max(span, 1e-9) / 1e6, 3),
        "steps_per_s": round(len(finished) / max(span, 1e-9), 1),
        "swapped_requests": int((~hit).sum()),
    }
    if refused:
        out["refused_requests"] = refused
    if hit.any() and not hit.all():
        out["p50_ms_resident"] = round(float(np.percentile(lat[hit], 50)), 3)
        out["p99_ms_resident"] = round(float(np.percentile(lat[hit], 99)), 3)
    return out


def latency_part(finished, cells_of):
    """One rank's raw results, for merge_parts on rank 0: latencies (ms),
    swapped flags, cells stepped, and the run's first arrival and last
    completion (the ranks' clocks start together at a barrier); refused
    requests only counted."""
    refused = sum(1 for r in finished if r.refused)
    finished = [r for r in finished if not r.refused]
    return {
        "refused": refused,
        "lat_ms": [(r.t_done - r.t_arrival) * 1e3 for r in finished],
        "swapped": [bool(r.swapped) for r in finished],
        "cells": int(sum(cells_of(r.world) for r in finished)),
        "t0": min((r.t_arrival for r in finished), default=0.0),
        "t1": max((r.t_done for r in finished), default=0.0),
    }


def merge_parts(parts):
    """latency_summary over several ranks' latency_part results: the
    percentiles of all requests, the throughput summed over the ranks."""
    lat = np.concatenate([np.asarray(p["lat_ms"], dtype=np.float64) for p in parts])
    hit = ~np.concatenate([np.asarray(p["swapped"], dtype=bool) for p in parts])
    refused = sum(p.get("refused", 0) for p in parts)
    if lat.size == 0:
        return {"requests": 0, "refused_requests": refused}
    parts = [p for p in parts if p["lat_ms"]]
    out = {
        "requests": int(lat.size),
        "p50_ms": round(float(np.percentile(lat, 50)), 3),
        "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "mean_ms": round(float(lat.mean()), 3),
        "mcells_per_s": round(sum(p["cells"] / max(p["t1"] - p["t0"], 1e-9) for p in parts) / 1e6, 3),
        "steps_per_s": round(sum(len(p["lat_ms"]) / max(p["t1"] - p["t0"], 1e-9) for p in parts), 1),
        "swapped_requests": int((~hit).sum()),
    }
    if refused:
        out["refused_requests"] = refused
    if hit.any() and not hit.all():
        out["p50_ms_resident"] = round(float(np.percentile(lat[hit], 50)), 3)
        out["p99_ms_resident"] = round(float(np.percentile(lat[hit], 99)), 3)
    return out
