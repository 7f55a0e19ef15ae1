"""The allocation-free entry point, wig_fluid_residual_norm2_noalloc.

It serves hosts that own all device memory and cannot let the library call
cudaMalloc (work recorded into a CUDA graph while it runs, a pre-reserved
pool under the host's own allocator, a real-time path).  It sums the FP64
squared norm of the pressure solve's residual into a device double the
caller passes, with its per-block scratch in a static device array instead
of an allocation.  Here it is checked against what the existing step entry
point reports for the same state, (rel_residual * b_norm)^2, on two calls in
a row, within the 1e-12 relative bar the tolerance tests use.  This file is
collected last, so a run that stops at the first failure has run the rest.
"""
import ctypes as C

import pytest

from worldinagrain_b200 import abi
from worldinagrain_b200 import world as W

from .common import params

pytestmark = pytest.mark.gpu

REL = 1e-12


def _entry():
    from worldinagrain_b200 import fluid
    f = fluid.lib().wig_fluid_residual_norm2_noalloc
    f.argtypes = [C.POINTER(abi.WorldDesc), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return fluid, f


# the step's forms: one kernel a reference pass, the fast form (the default),
# and the mixed-precision form, whose residual reaches cg through the fast
# form's write-back and may have been replaced by the true residual
FORMS = {"plain": abi.STEP_PLAIN, "fast": 0, "mixed": abi.STEP_MIXED}


@pytest.mark.parametrize("form", ["plain", "fast", "mixed"])
def test_noalloc_norm_matches_the_step_on_two_calls(form):
    import torch
    fluid, f = _entry()
    world = W.dam_break(64, 64)
    g = fluid.LiquidStep(world, W.element_table())
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    d = world.desc()
    for s in (1, 2):
        g.step(params(world, s), max_cycles=48, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS | FORMS[form],
               tolerance=1e-6)
        st = g.stats()
        b = g.buffers()
        rc = f(C.byref(d), b.field, b.blocks, b.cg, C.c_void_p(out.data_ptr()), None)
        assert rc == 0, fluid.lib().wig_fluid_last_error()
        torch.cuda.synchronize()
        got = float(out.item())
        want = (st.rel_residual * st.b_norm) ** 2
        assert want > 0.0
        assert abs(got - want) <= REL * want, (s, got, want)
    g.close()


def test_noalloc_refuses_worlds_past_its_maximum():
    fluid, f = _entry()
    d = abi.WorldDesc(1032, 1024, 4, 0)  # 129 x 128 blocks > WIG_NOALLOC_MAX_BLOCKS
    one = C.c_void_p(16)
    rc = f(C.byref(d), one, one, one, one, None)
    assert rc == -1
    assert b"at most 16384" in fluid.lib().wig_fluid_last_error()


def test_noalloc_norm_at_its_maximum_world():
    """A 1024x1024 world: 128 x 128 = 16384 blocks, exactly the static
    scratch's size (WIG_NOALLOC_MAX_BLOCKS)."""
    import torch
    fluid, f = _entry()
    world = W.disks_world(1024, 1024, seed=2)
    assert world.L["block_count"] == 16384
    g = fluid.LiquidStep(world, W.element_table())
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    d = world.desc()
    g.step(params(world, 1), max_cycles=64, flags=abi.STEP_TOLERANCE | abi.STEP_F64_DOTS, tolerance=1e-6)
    st = g.stats()
    b = g.buffers()
    rc = f(C.byref(d), b.field, b.blocks, b.cg, C.c_void_p(out.data_ptr()), None)
    assert rc == 0, fluid.lib().wig_fluid_last_error()
    torch.cuda.synchronize()
    want = (st.rel_residual * st.b_norm) ** 2
    assert want > 0.0
    assert abs(float(out.item()) - want) <= REL * want
    g.close()
