"""Writes tests/golden/oracle_steps.json: SHA-256 digests of the CPU oracle's
buffers after steps of small seeded worlds; and tests/golden/bodies_steps.json,
the same for the tank of synthetic free bodies with its body table and push
sums.

The reference ships no test vectors for the liquid step (its test/*.mjs
scripts are named in comments but absent), so these fixtures pin the oracle
itself: regenerate them only for a deliberate change of the oracle, and the
GPU tests compare the CUDA path with them too.  Grid buffers are digested
bit for bit; particles as the sorted rows of (motion, state with the sort
slot masked, affine), their order within a cell being an atomic's in the
reference.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from worldinagrain_b200 import abi  # noqa: E402
from worldinagrain_b200 import world as W  # noqa: E402
from tests.common import GRID, canonical_particles, mask_solve_scratch  # noqa: E402

CASES = [
    # name, builder, flags, max_cycles, steps recorded
    ("small_dam_ref", lambda: W.small_world(40, 32, seed=3, kind="dam"), 0, 16, (1, 4, 10)),
    ("small_obstacles_ref", lambda: W.small_world(40, 32, seed=3, kind="obstacles"), 0, 16, (1, 4, 10)),
    ("small_moving_tol", lambda: W.small_world(40, 32, seed=3, kind="moving"),
     abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, 48, (1, 4, 10)),
    ("dam64_tol", lambda: W.dam_break(64, 64), abi.STEP_TOLERANCE, 48, (1, 6)),
]


BODY_CASES = [
    # name, liquid, flags, max_cycles, steps recorded
    ("bodies_water_tol", abi.WATER, abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, 64, (1, 3, 6)),
    ("bodies_water_ref", abi.WATER, 0, 16, (1, 4)),
    ("bodies_mud_tol", W.MUD, abi.STEP_TOLERANCE | abi.STEP_F64_DOTS | abi.STEP_VISCOUS, 64, (1, 4)),
]


def digest(a):
    return hashlib.sha256(memoryview(a).cast("B")).hexdigest()


def world_digests(world):
    out = {name: digest(getattr(world, name)) for name in GRID}
    # the same with the solve's scratch words left out (the fast form's check)
    for name in ("counters", "field"):
        out[name + "_observable"] = digest(mask_solve_scratch(world, name, getattr(world, name)))
    for which in ("sorted", "parts"):
        out[which] = digest(canonical_particles(world, which).astype("<u8").copy())
        out[which + "_count"] = int(getattr(world, which)[0])
    return out


def run_case(builder, flags, max_cycles, record):
    world = builder()
    o = Oracle(world, W.element_table())
    got = {}
    for s in range(1, max(record) + 1):
        P = W.make_params(world, frame=s, seed=0x1234, earth_g=world.config["earth_g"])
        st = o.step(P, max_cycles=max_cycles, flags=flags, tolerance=1e-6)
        if s in record:
            d = world_digests(world)
            d["cycles"] = int(st.cycles)
            got[str(s)] = d
    return got


def run_body_case(liquid, flags, max_cycles, record):
    world, bodies = W.bodies_world(liquid=liquid)
    o = Oracle(world, W.body_element_table(), bodies)
    got = {}
    for s in range(1, max(record) + 1):
        P = W.make_params(world, frame=s, seed=0x1234, earth_g=world.config["earth_g"])
        bodies.stamp_step(s - 1)
        W.send_aside(world, bodies, s)
        st = o.step(P, max_cycles=max_cycles, flags=flags, tolerance=1e-6)
        if s in record:
            d = world_digests(world)
            d["motion"] = digest(bodies.motion)
            d["pushes"] = digest(bodies.pushes)
            d["cycles"] = int(st.cycles)
            got[str(s)] = d
    return got


def main():
    fixtures = {}
    for name, builder, flags, max_cycles, record in CASES:
        fixtures[name] = {"flags": flags, "max_cycles": max_cycles, "steps": run_case(builder, flags, max_cycles, record)}
    with open(os.path.join(HERE, "oracle_steps.json"), "w") as f:
        json.dump(fixtures, f, indent=1, sort_keys=True)
    bodies = {}
    for name, liquid, flags, max_cycles, record in BODY_CASES:
        bodies[name] = {"flags": flags, "max_cycles": max_cycles,
                        "steps": run_body_case(liquid, flags, max_cycles, record)}
    with open(os.path.join(HERE, "bodies_steps.json"), "w") as f:
        json.dump(bodies, f, indent=1, sort_keys=True)
    print("wrote", len(fixtures) + len(bodies), "cases")


if __name__ == "__main__":
    main()
