"""Each form's pressure and velocity against an FP64 solve of the same
system, per config: the dam 256x256 world, the disks 1024x1024 world and
a world of two liquids of different densities, each after three steps.
The FP64 solve is the oracle's CG of the same operator and right-hand side
to a 1e-12 relative residual; the forms stop at 1e-6. The velocity error is that of the projected faces: the oracle's
project pass run once with the form's pressure and once with the FP64 one
(the form's drift potential in both), over the faces it projects. The
plain and fast forms are the oracle's bits, so their errors are the FP32
solve's; the mixed form stores its coarse operator in binary16. Each case
prints its errors (pytest -s shows them)."""
import numpy as np
import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

pytestmark = pytest.mark.gpu

TOL = abi.STEP_TOLERANCE | abi.STEP_F64_DOTS
FORMS = (("plain", abi.STEP_PLAIN | TOL), ("fast", TOL), ("mixed", abi.STEP_MIXED | TOL))
PRE = ("SYNC", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER", "SEAL_JOIN",
       "SEAL_ANCHOR", "CLASSIFY", "SET_FACES", "UNPRESS", "DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR")
# (name, world, bound on the pressure's and the velocity's relative L2 error)
CASES = (
    ("dam 256x256", lambda: W.dam_break(256, 256, seed=1), 1e-4),
    ("disks 1024x1024", lambda: W.disks_world(1024, 1024, seed=2), 1e-3),
    # water beside a denser liquid: coarse densities and coefficients that
    # binary16 rounds (with one density they are exact in it)
    ("two liquids 192x160", lambda: W.two_liquids(192, 160, seed=5), 1e-4),
)


def _params(world, step):
    return W.make_params(world, frame=step, seed=2, earth_g=world.config["earth_g"])


def _faces(world):
    F = world.L["face_count"]
    return world.field[8 * world.C: 8 * world.C + 4 * F].reshape(F, 4)


def _projected(probe, P, pressure, drift):
    """The oracle's project pass on a copy of the probe (the step's passes
    up to the solve done) with the given pressure and drift potential."""
    from oracle.oracle import Oracle
    q = probe.copy()
    fc = q.field_cells()
    fc[:, 0, 0] = pressure
    fc[:, 1, 0] = drift
    Oracle(q, W.element_table()).pass_(P, "PROJECT")
    return _faces(q)


@pytest.mark.parametrize("case", [c[0] for c in CASES])
def test_forms_against_the_fp64_solve(case):
    from oracle.oracle import Oracle
    from worldinagrain_b200 import fluid
    _, builder, bound = next(c for c in CASES if c[0] == case)
    world = builder()
    g = fluid.LiquidStep(world, W.element_table())
    for s in range(1, 4):
        g.step(_params(world, s), max_cycles=64, flags=TOL, tolerance=1e-6)
    g.download()
    g.close()
    P = _params(world, 4)
    probe = world.copy()
    po = Oracle(probe, W.element_table())
    for name in PRE:
        po.pass_(P, name)
    x64, _, rel = po.solve_f64(P, rel_tol=1e-12)
    assert rel <= 1e-12
    fluid_ = probe.field_cells()[:, 0, 2] > 0
    pressures = {}
    for form, flags in FORMS:
        w = world.copy()
        h = fluid.LiquidStep(w, W.element_table())
        h.step(P, max_cycles=64, flags=flags | abi.STEP_SHIFTED_SET, tolerance=1e-6)
        st = h.stats()
        h.download()
        h.close()
        p = w.field_cells()[:, 0, 0].copy()
        drift = w.field_cells()[:, 1, 0].copy()
        pressures[form] = p
        ep = np.linalg.norm(p[fluid_].astype(np.float64) - x64[fluid_]) / np.linalg.norm(x64[fluid_])
        ua = _projected(probe, P, p, drift)
        ub = _projected(probe, P, np.where(fluid_, x64, p).astype(np.float32), drift)
        on = ub[:, 2] == 2.0  # the faces the pass projected
        eu = (np.linalg.norm(ua[on, 0].astype(np.float64) - ub[on, 0]) /
              np.linalg.norm(ub[on, 0].astype(np.float64)))
        print(f"\n{case} {form}: pressure {ep:.3e}, velocity {eu:.3e} relative L2 against the FP64 solve; "
              f"{st.cycles} iterations, residual {st.rel_residual:.2e}")
        assert st.rel_residual <= 1e-6
        assert ep < bound and eu < bound, (form, ep, eu)
    # the FP32 forms are the same solve
    assert np.array_equal(pressures["plain"], pressures["fast"])
