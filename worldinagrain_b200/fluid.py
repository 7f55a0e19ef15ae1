"""Host side of the liquid step: the reference's Simulation liquid interface
(js/sim.js:741-843 allocation, :2466-2612 encodeFluid, :1882-1900
readReport) over the C ABI of libwig_fluid.so.

There is no CPU path here: a missing library or device raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libwig_fluid.so")

_lib = None

FUNCS = {
    "wig_fluid_abi_version": ([], C.c_uint32),
    "wig_fluid_last_error": ([], C.c_char_p),
    "wig_fluid_layout": ([C.POINTER(abi.WorldDesc), C.POINTER(abi.WorldLayout)], C.c_int),
    "wig_fluid_create": ([C.POINTER(abi.WorldDesc), C.POINTER(abi.Elem), C.c_uint32, C.POINTER(C.c_void_p)], C.c_int),
    "wig_fluid_bind": ([C.c_void_p, C.POINTER(abi.Buffers)], C.c_int),
    "wig_fluid_bind_bodies": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "wig_fluid_buffers_of": ([C.c_void_p, C.POINTER(abi.Buffers)], C.c_int),
    "wig_fluid_step": ([C.c_void_p, C.POINTER(abi.Params), C.c_uint32, C.c_uint32, C.c_double, C.c_void_p], C.c_int),
    "wig_fluid_dispatch": ([C.c_void_p, C.POINTER(abi.Params), C.c_int, C.c_uint32, C.c_uint32, C.c_void_p], C.c_int),
    "wig_fluid_upload": ([C.c_void_p, C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p], C.c_int),
    "wig_fluid_download": ([C.c_void_p, C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p], C.c_int),
    "wig_fluid_read_stats": ([C.c_void_p, C.POINTER(abi.Stats)], C.c_int),
    "wig_fluid_step_profile": ([C.c_void_p, C.POINTER(abi.Params), C.c_uint32, C.c_uint32, C.c_double, C.c_void_p,
                                C.POINTER(C.c_float), C.POINTER(C.c_uint32)], C.c_int),
    "wig_fluid_destroy": ([C.c_void_p], None),
    "wig_batch_world_bytes": ([C.POINTER(abi.WorldDesc), C.POINTER(C.c_uint64)], C.c_int),
    "wig_batch_create": ([C.POINTER(abi.WorldDesc), C.c_uint32, C.POINTER(abi.Elem), C.c_uint32, C.POINTER(C.c_void_p)],
                         C.c_int),
    "wig_batch_worlds": ([C.c_void_p], C.c_uint32),
    "wig_batch_layout": ([C.c_void_p, C.c_uint32, C.POINTER(abi.WorldLayout)], C.c_int),
    "wig_batch_buffers_of": ([C.c_void_p, C.c_uint32, C.POINTER(abi.Buffers)], C.c_int),
    "wig_batch_upload": ([C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p], C.c_int),
    "wig_batch_download": ([C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p], C.c_int),
    "wig_batch_step": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(abi.Params),
                        C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32, C.c_double, C.c_void_p], C.c_int),
    "wig_batch_read_stats": ([C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(abi.Stats)], C.c_int),
    "wig_batch_step_profile": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(abi.Params),
                                C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32, C.c_double, C.c_void_p,
                                C.POINTER(C.c_float), C.POINTER(C.c_uint32)], C.c_int),
    "wig_batch_destroy": ([C.c_void_p], None),
    "wig_batch_set_launch": ([C.c_void_p, C.c_uint32, C.c_uint32], C.c_int),
    "wig_fluid_set_launch": ([C.c_void_p, C.c_uint32, C.c_uint32], C.c_int),
    "wig_fluid_get_launch": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)], C.c_int),
    "wig_batch_get_launch": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)], C.c_int),
    "wig_fluid_set_wait_limits": ([C.c_uint32, C.c_uint32], C.c_int),
}


class WigError(RuntimeError):
    pass


class NotConverged(WigError):
    """WIG_E_NOT_CONVERGED from a stats read: a tolerance-form solve stopped
    after max_cycles above its tolerance.  The step itself is complete;
    `stats` holds the report (one Stats, or a list for a batch)."""

    def __init__(self, msg, stats):
        super().__init__(msg)
        self.stats = stats


E_NOT_CONVERGED = -5


def lib(path=None):
    """Loads libwig_fluid.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise WigError(f"libwig_fluid.so not built ({p}); run worldinagrain_b200/build.py")
        L = C.CDLL(p)
        for name, (args, res) in FUNCS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        if L.wig_fluid_abi_version() != abi.ABI_VERSION:
            raise WigError("libwig_fluid.so ABI version mismatch")
        _lib = L
    return _lib


def check(rc, what):
    if rc != 0:
        msg = lib().wig_fluid_last_error().decode(errors="replace")
        raise WigError(f"{what}: {abi.ERRORS.get(rc, rc)}: {msg}")


class LiquidStep:
    """One world's liquid on the GPU: its buffers resident in device memory,
    stepped by wig_fluid_step.  `stream` is a cudaStream_t as an int (0: the
    legacy stream)."""

    def __init__(self, world, elems, stream=0):
        self.world = world
        self.elems = elems
        self.stream = C.c_void_p(stream or None)
        L = lib()
        h = C.c_void_p()
        d = world.desc()
        check(L.wig_fluid_create(C.byref(d), elems, len(elems), C.byref(h)), "wig_fluid_create")
        self.h = h
        check(L.wig_fluid_bind(h, None), "wig_fluid_bind")
        self.upload()

    def close(self):
        if getattr(self, "h", None):
            lib().wig_fluid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, world=None):
        w = world or self.world
        for k, name in enumerate(abi.BUFFER_NAMES):
            arr = np.ascontiguousarray(getattr(w, name))
            check(lib().wig_fluid_upload(self.h, k, arr.ctypes.data, 0, arr.nbytes, self.stream), f"upload {name}")

    def download(self, world=None, names=abi.BUFFER_NAMES):
        w = world or self.world
        for name in names:
            k = abi.BUFFER_NAMES.index(name)
            arr = getattr(w, name)
            assert arr.flags["C_CONTIGUOUS"]
            check(lib().wig_fluid_download(self.h, k, arr.ctypes.data, 0, arr.nbytes, self.stream), f"download {name}")
        return w

    def buffers(self):
        b = abi.Buffers()
        check(lib().wig_fluid_buffers_of(self.h, C.byref(b)), "buffers_of")
        return b

    def bind_bodies(self, bodies):
        """Binds a free-body table, push sums and bodies' buffer
        (world.Bodies) in device memory of their own (bindings 12, 16 and
        14, js/sim.js:1159); the steps after couple the bodies into the
        solve.  None unbinds them."""
        import torch
        if bodies is None:
            check(lib().wig_fluid_bind_bodies(self.h, None, None, None), "wig_fluid_bind_bodies")
            self._bodies = None
            return
        devs = tuple(torch.from_numpy(a.view(np.int32).copy()).to("cuda")
                     for a in (bodies.motion, bodies.pushes, bodies.stamps))
        torch.cuda.synchronize()
        check(lib().wig_fluid_bind_bodies(self.h, *(C.c_void_p(t.data_ptr()) for t in devs)), "wig_fluid_bind_bodies")
        self._bodies = devs

    def upload_bodies(self, bodies):
        """bodies' table, push sums and stamps copied into the bound device
        buffers."""
        import torch
        for t, a in zip(self._bodies, (bodies.motion, bodies.pushes, bodies.stamps)):
            t.copy_(torch.from_numpy(a.view(np.int32).copy()))
        torch.cuda.synchronize()

    def download_bodies(self, bodies):
        """The bound body table and push sums copied back into bodies (the
        stamps the step only reads)."""
        import torch
        motion, pushes, _ = self._bodies
        torch.cuda.synchronize()
        bodies.motion[:] = motion.cpu().numpy().view(np.uint32)
        bodies.pushes[:] = pushes.cpu().numpy().view(np.uint32)
        return bodies

    def step(self, P, max_cycles=abi.FLUID_CYCLES, flags=0, tolerance=1e-6):
        check(lib().wig_fluid_step(self.h, C.byref(P), max_cycles, flags, tolerance, self.stream), "wig_fluid_step")

    def step_profile(self, P, max_cycles=abi.FLUID_CYCLES, flags=0, tolerance=1e-6):
        """One step launched pass by pass with CUDA events around each:
        {pass name: (ms, launches)}."""
        ms = (C.c_float * abi.PROFILE_SLOTS)()
        calls = (C.c_uint32 * abi.PROFILE_SLOTS)()
        check(lib().wig_fluid_step_profile(self.h, C.byref(P), max_cycles, flags, tolerance, self.stream, ms, calls),
              "wig_fluid_step_profile")
        return {abi.PROFILE_NAMES[k]: (ms[k], calls[k]) for k in range(abi.PROFILE_SLOTS) if calls[k]}

    def set_launch(self, knob, value):
        """One launch shape of the fast form (abi.LAUNCH_KNOBS); no result
        changes."""
        k = abi.LAUNCH_KNOBS.get(knob, knob)
        check(lib().wig_fluid_set_launch(self.h, k, int(value)), f"wig_fluid_set_launch {knob}")

    def get_launch(self, knob):
        k = abi.LAUNCH_KNOBS.get(knob, knob)
        v = C.c_uint32()
        check(lib().wig_fluid_get_launch(self.h, k, C.byref(v)), f"wig_fluid_get_launch {knob}")
        return v.value

    def launch_shapes(self):
        return {name: self.get_launch(name) for name in abi.LAUNCH_KNOBS}

    def dispatch(self, P, name, level=0, cycle=0):
        check(lib().wig_fluid_dispatch(self.h, C.byref(P), abi.PASS[name], level, cycle, self.stream), f"dispatch {name}")

    def stats(self, unconverged_ok=False):
        """The last step's report (wig_fluid_read_stats).  A solve short of
        its tolerance raises NotConverged unless unconverged_ok."""
        st = abi.Stats()
        rc = lib().wig_fluid_read_stats(self.h, C.byref(st))
        return _stats_or_raise(rc, st, unconverged_ok, "wig_fluid_read_stats")


def set_wait_limits(loop_limit=0, spin_limit=0):
    """Lowers the device's retry and barrier-wait bounds on the current
    device (0: the default) so a failure-path test sees them run out."""
    check(lib().wig_fluid_set_wait_limits(loop_limit, spin_limit), "wig_fluid_set_wait_limits")


def _stats_or_raise(rc, stats, unconverged_ok, what):
    if rc == E_NOT_CONVERGED:
        if unconverged_ok:
            return stats
        msg = lib().wig_fluid_last_error().decode(errors="replace")
        raise NotConverged(f"{what}: WIG_E_NOT_CONVERGED: {msg}", stats)
    check(rc, what)
    return stats


def world_bytes(width, height, liquid_per_cell=4, capacity=0):
    """Device bytes a world of this shape holds in a batch."""
    d = abi.WorldDesc(width, height, liquid_per_cell, capacity)
    out = C.c_uint64()
    check(lib().wig_batch_world_bytes(C.byref(d), C.byref(out)), "wig_batch_world_bytes")
    return out.value


def _u32s(seq):
    seq = list(seq)
    return (C.c_uint32 * max(len(seq), 1))(*seq)


class Batch:
    """Many worlds resident on the GPU in one packed allocation, stepped
    together: each pass one launch over all the worlds listed (the
    reference's Simulation holds one world; this has no counterpart there).
    `worlds` are World objects (their numpy buffers uploaded at creation)."""

    LANES = 2

    def __init__(self, worlds, elems):
        self.worlds = list(worlds)
        self.elems = elems
        L = lib()
        descs = (abi.WorldDesc * len(self.worlds))(*[w.desc() for w in self.worlds])
        h = C.c_void_p()
        check(L.wig_batch_create(descs, len(self.worlds), elems, len(elems), C.byref(h)), "wig_batch_create")
        self.h = h
        for k in range(len(self.worlds)):
            self.upload(k)

    def close(self):
        if getattr(self, "h", None):
            lib().wig_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.worlds)

    def upload(self, k, world=None, stream=0):
        w = world or self.worlds[k]
        for which, name in enumerate(abi.BUFFER_NAMES):
            arr = np.ascontiguousarray(getattr(w, name))
            check(lib().wig_batch_upload(self.h, k, which, arr.ctypes.data, 0, arr.nbytes, C.c_void_p(stream or None)),
                  f"upload {name} of world {k}")

    def download(self, k, world=None, names=abi.BUFFER_NAMES, stream=0):
        w = world or self.worlds[k]
        for name in names:
            which = abi.BUFFER_NAMES.index(name)
            arr = getattr(w, name)
            assert arr.flags["C_CONTIGUOUS"]
            check(lib().wig_batch_download(self.h, k, which, arr.ctypes.data, 0, arr.nbytes, C.c_void_p(stream or None)),
                  f"download {name} of world {k}")
        return w

    def buffers(self, k):
        b = abi.Buffers()
        check(lib().wig_batch_buffers_of(self.h, k, C.byref(b)), "wig_batch_buffers_of")
        return b

    def step(self, ids, params, world_flags=None, max_cycles=abi.FLUID_CYCLES, flags=0, tolerance=1e-6, lane=0,
             stream=0):
        """One step of the worlds `ids` (params[i] for ids[i]), asynchronous.
        ids, params and world_flags may be prebuilt ctypes arrays."""
        n = len(ids)
        ids_a = ids if isinstance(ids, C.Array) else _u32s(ids)
        P = params if isinstance(params, C.Array) else (abi.Params * n)(*params)
        wf = None
        if world_flags is not None:
            wf = world_flags if isinstance(world_flags, C.Array) else _u32s(world_flags)
        check(lib().wig_batch_step(self.h, lane, ids_a, n, P, wf, max_cycles, flags, tolerance,
                                   C.c_void_p(stream or None)), "wig_batch_step")

    def step_profile(self, ids, params, world_flags=None, max_cycles=abi.FLUID_CYCLES, flags=0, tolerance=1e-6,
                     lane=0, stream=0):
        ids = list(ids)
        P = (abi.Params * len(ids))(*params)
        wf = _u32s(world_flags) if world_flags is not None else None
        ms = (C.c_float * abi.PROFILE_SLOTS)()
        calls = (C.c_uint32 * abi.PROFILE_SLOTS)()
        check(lib().wig_batch_step_profile(self.h, lane, _u32s(ids), len(ids), P, wf, max_cycles, flags, tolerance,
                                           C.c_void_p(stream or None), ms, calls), "wig_batch_step_profile")
        return {abi.PROFILE_NAMES[k]: (ms[k], calls[k]) for k in range(abi.PROFILE_SLOTS) if calls[k]}

    def stats(self, ids, unconverged_ok=False):
        """The worlds' reports (wig_batch_read_stats); NotConverged as for
        LiquidStep.stats."""
        ids = list(ids)
        out = (abi.Stats * len(ids))()
        rc = lib().wig_batch_read_stats(self.h, _u32s(ids), len(ids), out)
        return _stats_or_raise(rc, list(out), unconverged_ok, "wig_batch_read_stats")

    def set_launch(self, knob, value):
        """One launch shape (abi.LAUNCH_KNOBS: a name or its number); no
        result changes."""
        k = abi.LAUNCH_KNOBS.get(knob, knob)
        check(lib().wig_batch_set_launch(self.h, k, int(value)), f"wig_batch_set_launch {knob}")

    def get_launch(self, knob):
        k = abi.LAUNCH_KNOBS.get(knob, knob)
        v = C.c_uint32()
        check(lib().wig_batch_get_launch(self.h, k, C.byref(v)), f"wig_batch_get_launch {knob}")
        return v.value

    def launch_shapes(self):
        return {name: self.get_launch(name) for name in abi.LAUNCH_KNOBS}
