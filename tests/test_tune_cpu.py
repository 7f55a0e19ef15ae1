"""The launch-shape autotuner's choices, over a fake batch whose profiled
steps cost what a table says: each knob ends at its cheapest candidate,
tried in order, each knob tuned with the earlier knobs' choices in place,
and a cost that drifts from step to step does not decide the choice."""
from worldinagrain_b200 import tune


class FakeBatch:
    def __init__(self, costs):
        self.shapes = {"coarse_cells": 4096, "level_per_sm": 8, "cg_per_sm": 8, "relax_per_sm": 16}
        self.costs = costs  # knob -> value -> ms per iteration of its slots
        self.log = []

    def get_launch(self, name):
        return self.shapes[name]

    def set_launch(self, name, value):
        self.shapes[name] = value
        self.log.append((name, value))

    def launch_shapes(self):
        return dict(self.shapes)

    def step(self):
        iters = 7
        prof = {"F_LOOP": (0.1, iters)}
        for name, _, slots in tune.KNOBS:
            share = self.costs[name][self.shapes[name]] * iters / len(slots)
            for s in slots:
                ms, n = prof.get(s, (0.0, 0))
                prof[s] = (ms + share, n + iters)
        return prof


def test_each_knob_ends_at_its_cheapest_candidate():
    # per knob, its candidates' costs: the second cheapest for the first
    # knob, the first for the second, and so on
    costs, want = {}, {}
    for j, (name, cands, _) in enumerate(tune.KNOBS):
        cheap = cands[(j + 1) % len(cands)]
        costs[name] = {v: (1.0 if v == cheap else 2.0 + 0.1 * i) for i, v in enumerate(cands)}
        want[name] = cheap
    b = FakeBatch(costs)
    shapes, trials = tune.autotune(b, b.step)
    assert shapes == want
    assert [v for v, _ in trials["coarse_cells"]] == list(tune.KNOBS[0][1])
    assert len(b.log) == tune.steps_needed() + len(tune.KNOBS)


def test_cost_is_per_iteration_and_none_without_iterations():
    assert tune.cost({"F_LOOP": (0.0, 4), "F_RELAX": (8.0, 8)}, ("F_RELAX",)) == 2.0
    assert tune.cost({"F_RELAX": (8.0, 8)}, ("F_RELAX",)) is None


def test_no_iteration_keeps_the_current_shape():
    class Idle(FakeBatch):
        def step(self):
            return {}
    b = Idle({})
    shapes, _ = tune.autotune(b, b.step)
    assert shapes == {"coarse_cells": 4096, "level_per_sm": 8, "cg_per_sm": 8, "relax_per_sm": 16}


def test_a_drift_over_the_steps_weighs_the_same_on_every_candidate():
    """The steps' cost falls by 0.05 ms an iteration a step (the worlds move
    on); the first candidate is cheapest by 0.1. One pass in order would
    pick the last candidate; the two passes pick the first."""
    name, cands, slots = tune.KNOBS[0]

    class Drifting(FakeBatch):
        def __init__(self):
            super().__init__({})
            self.n = 0

        def step(self):
            c = (1.0 if self.shapes[name] == cands[0] else 1.1) - 0.05 * self.n
            self.n += 1
            return {"F_LOOP": (0.1, 7), slots[0]: (c * 7, 7)}

    b = Drifting()
    shapes, trials = tune.autotune(b, b.step, knobs=(tune.KNOBS[0],))
    assert shapes[name] == cands[0] and b.n == 2 * len(cands)
    b = Drifting()
    shapes, _ = tune.autotune(b, b.step, knobs=(tune.KNOBS[0],), passes=1)
    assert shapes[name] == cands[-1]


def test_a_refused_candidate_is_left_out():
    """A batch of several worlds refuses coarse cells above 4096 (the
    single world's cluster range): that candidate gets no cost and no step,
    and the choice falls among the others."""
    from worldinagrain_b200.fluid import WigError

    class Several(FakeBatch):
        def set_launch(self, name, value):
            if name == "coarse_cells" and value > 4096:
                raise WigError("launch knob value out of range")
            super().set_launch(name, value)
    costs = {name: {v: 1.0 + 0.1 * i for i, v in enumerate(c)} for name, c, _ in tune.KNOBS}
    b = Several(costs)
    shapes, trials = tune.autotune(b, b.step)
    assert dict(trials["coarse_cells"])[16384] is None
    assert shapes["coarse_cells"] == 4096
    assert all(v <= 4096 for n, v in b.log if n == "coarse_cells")


def test_the_profiled_steps_launch_floor_is_not_counted():
    """A candidate with fewer launches is not credited with the profiled
    step's per-launch overhead (FLOOR_SHARE of the loop-start kernel's time
    a launch): 6 launches of 0.02 ms against 8 of 0.016 ms, floor 0.005 ms
    of the loop start's 0.01, cost 0.09 against 0.088 ms; counting the whole
    time would pick the first."""
    assert tune.FLOOR_SHARE == 0.5
    few = {"F_LOOP": (0.01, 1), "F_COARSE": (0.12, 6)}
    many = {"F_LOOP": (0.01, 1), "F_COARSE": (0.128, 8)}
    assert abs(tune.cost(few, ("F_COARSE",)) - 0.09) < 1e-12
    assert abs(tune.cost(many, ("F_COARSE",)) - 0.088) < 1e-12


def test_the_current_shape_stays_unless_clearly_beaten():
    """A candidate 2% cheaper than the batch's own shape does not replace it
    (the profiled steps' spread is about 3%); one 5% cheaper does."""
    name, cands, slots = tune.KNOBS[1]  # level_per_sm, current 8
    for cheaper, want in ((0.98, 8), (0.95, cands[0])):
        costs = {n: {v: 1.0 for v in c} for n, c, _ in tune.KNOBS}
        costs[name][cands[0]] = cheaper
        b = FakeBatch(costs)
        shapes, _ = tune.autotune(b, b.step, knobs=(tune.KNOBS[1],))
        assert shapes[name] == want
