"""Launch-shape autotuner of a batch of worlds.

A batch steps its worlds with one launch a pass; how those launches are
shaped is the batch's choice (include/wig_batch.h, wig_launch_knob):

- coarse_cells: from which level the coarse kernel takes over a world's
  V-cycle (the depth of its on-chip part; above 4096, a single world's on a
  cluster of CTAs, a value a batch of several worlds refuses and the tuner
  leaves out);
- level_per_sm, cg_per_sm, relax_per_sm: the CTAs a multiprocessor of the
  level tile kernels, the CG kernels and the fine relaxation.

No knob changes a result bit, so the tuner tunes on the batch's own steps.
Each candidate runs profiled steps (device timestamps around every launch).
Its cost is the time, per solver iteration, of the kernels the knob shapes.
The cheapest candidate is kept. Knobs are tuned one after another, each
given the choices made before it.

Successive steps are different steps of the worlds: their solves take
other iterations, and a batch's worlds stop iterating at other times, so a
step's cost per iteration drifts as the worlds move on. The candidates are
therefore tried in two passes, in order and then in reverse, and each
candidate's cost is taken over both of its steps: a drift that is linear
over the knob's steps weighs the same on every candidate.
"""

from .fluid import WigError

# A candidate replaces the batch's shape only when cheaper by more than this
# share: the profiled steps differ by about that much from step to step.
MARGIN = 0.03
# The share of the loop-start kernel's profiled time a launch that is the
# profiling's own overhead (the rest is the launch's cost in the graph too).
# On the 1024x1024 world the whole of it ranked coarse cells 512 first, by
# 4%, which the graph ran 2% slower than 1024 (166.8 against 170.5
# Mcells/s); half of it ranks them as the graph does.
FLOOR_SHARE = 0.5

KNOBS = (
    ("coarse_cells", (16384, 4096, 2048, 1024, 512), ("F_RESTRICT", "F_PROLONG", "F_COARSE")),
    ("level_per_sm", (4, 8, 16, 32), ("F_RESTRICT", "F_PROLONG")),
    ("cg_per_sm", (2, 4, 8, 16, 32), ("F_RHO_BETA", "F_APPLY_ALPHA", "F_UPDATE")),
    ("relax_per_sm", (16, 32, 64), ("F_RELAX",)),
)


def cost(profile, slots):
    """Milliseconds per solver iteration of `slots` in one profiled step
    (profile: slot name -> (ms, launches)); None when no iteration ran."""
    ms, iters = slot_time(profile, slots)
    return ms / iters if iters else None


def slot_time(profile, slots):
    """(milliseconds of `slots`, solver iterations) of one profiled step.

    A profiled step launches pass by pass with events around each launch,
    which costs every launch a floor the graph does not pay: the loop-start
    kernel's time a launch (one warp of bookkeeping) measures it. Each slot
    is counted less that floor for each of its launches, so a candidate
    with fewer, longer launches (a deeper coarse kernel) is not credited
    with the profiling's overhead. Measured on the 1024x1024 world: the
    eager step put the cluster coarse kernel (coarse cells 16384) 3% ahead
    of the one-CTA kernel at 4096; the graph ran it 2% behind. Only
    FLOOR_SHARE of the loop-start kernel's time is taken out: the rest is
    the launch's cost in the graph as well."""
    loop_ms, iters = profile.get("F_LOOP", (0.0, 0))
    floor = FLOOR_SHARE * loop_ms / iters if iters else 0.0
    ms = 0.0
    for s in slots:
        t, n = profile.get(s, (0.0, 0))
        ms += max(t - n * floor, 0.0)
    return ms, iters


def autotune(batch, step, knobs=KNOBS, passes=2):
    """Tune `batch` (fluid.Batch or anything with get_launch, set_launch and
    launch_shapes) on its own steps: step() runs one profiled step of the
    caller's worlds and returns Batch.step_profile's dict. Each candidate is
    stepped once a pass, the passes alternating in order and in reverse.
    Returns the chosen shapes and, per knob, the (value, cost) of each
    candidate in the knob's order. The batch keeps the chosen shapes."""
    trials = {}
    for name, candidates, slots in knobs:
        keep = batch.get_launch(name)
        ms = {v: 0.0 for v in candidates}
        its = {v: 0 for v in candidates}
        refused = set()
        for p in range(passes):
            for v in (candidates if p % 2 == 0 else tuple(reversed(candidates))):
                if v in refused:
                    continue
                try:
                    batch.set_launch(name, v)
                except WigError:
                    # out of this batch's range (coarse cells above 4096 on
                    # more than one world): no cost
                    refused.add(v)
                    continue
                t, n = slot_time(step(), slots)
                ms[v] += t
                its[v] += n
        rows = [(v, ms[v] / its[v] if its[v] else None) for v in candidates]
        best_v, best_c = keep, None
        for v, c in rows:
            if c is not None and (best_c is None or c < best_c):
                best_v, best_c = v, c
        # the shape the batch had stays unless a candidate beats it by more
        # than the profiled steps' spread
        kept = dict(rows).get(keep)
        if kept is not None and best_c is not None and best_c > (1.0 - MARGIN) * kept:
            best_v = keep
        batch.set_launch(name, best_v)
        trials[name] = rows
    return batch.launch_shapes(), trials


def steps_needed(knobs=KNOBS, passes=2):
    """Profiled steps autotune runs."""
    return passes * sum(len(c) for _, c, _ in knobs)
