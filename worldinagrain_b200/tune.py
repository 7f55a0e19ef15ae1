"""Launch-shape autotuner of a batch of worlds.

A batch steps its worlds with one launch a pass; how those launches are
shaped is the batch's choice (include/wig_batch.h, wig_launch_knob):

- coarse_cells: from which level the one-CTA coarse kernel takes over a
  world's V-cycle (the depth of its on-chip part);
- level_per_sm, cg_per_sm, relax_per_sm: the CTAs a multiprocessor of the
  level tile kernels, the CG kernels and the fine relaxation.

No knob changes a result bit, so the tuner tunes on the batch's own steps.
Each candidate runs one profiled step (device timestamps around every
launch). Its cost is the time, per solver iteration, of the kernels the
knob shapes. The cheapest candidate is kept. Knobs are tuned one after
another, each given the choices made before it.
"""

KNOBS = (
    ("coarse_cells", (4096, 2048, 1024, 512), ("F_RESTRICT", "F_PROLONG", "F_COARSE")),
    ("level_per_sm", (4, 8, 16, 32), ("F_RESTRICT", "F_PROLONG")),
    ("cg_per_sm", (2, 4, 8, 16, 32), ("F_RHO_BETA", "F_APPLY_ALPHA", "F_UPDATE")),
    ("relax_per_sm", (16, 32, 64), ("F_RELAX",)),
)


def cost(profile, slots):
    """Milliseconds per solver iteration of `slots` in one profiled step
    (profile: slot name -> (ms, launches)); None when no iteration ran."""
    iters = profile.get("F_LOOP", (0.0, 0))[1]
    if not iters:
        return None
    return sum(profile.get(s, (0.0, 0))[0] for s in slots) / iters


def autotune(batch, step, knobs=KNOBS):
    """Tune `batch` (fluid.Batch or anything with get_launch, set_launch and
    launch_shapes) on its own steps: step() runs one profiled step of the
    caller's worlds and returns Batch.step_profile's dict. Returns the chosen
    shapes and, per knob, the (value, cost) of each candidate tried. The
    batch keeps the chosen shapes."""
    trials = {}
    for name, candidates, slots in knobs:
        best_v, best_c = batch.get_launch(name), None
        rows = []
        for v in candidates:
            batch.set_launch(name, v)
            c = cost(step(), slots)
            rows.append((v, c))
            if c is not None and (best_c is None or c < best_c):
                best_v, best_c = v, c
        batch.set_launch(name, best_v)
        trials[name] = rows
    return batch.launch_shapes(), trials


def steps_needed(knobs=KNOBS):
    """Profiled steps autotune runs."""
    return sum(len(c) for _, c, _ in knobs)
