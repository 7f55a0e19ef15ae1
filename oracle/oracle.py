"""TEST INFRASTRUCTURE: ctypes front of the CPU oracle (oracle/wig_oracle.cpp).

The oracle restates the reference's liquid passes on the CPU; it is the
checker the CUDA path is compared with.  Only tests/, the smoke check and
bench.py's CPU-baseline leg load it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from worldinagrain_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libwig_oracle.so")
_lib = None


def build():
    """Compile the oracle (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.wo_layout.argtypes = [C.POINTER(abi.WorldDesc), C.POINTER(abi.WorldLayout)]
        L.wo_pass.argtypes = [C.POINTER(abi.WorldDesc), C.POINTER(abi.Params), C.POINTER(abi.Elem), C.c_uint32,
                              C.POINTER(abi.Buffers), C.c_int, C.c_uint32, C.c_uint32]
        L.wo_step.argtypes = [C.POINTER(abi.WorldDesc), C.POINTER(abi.Params), C.POINTER(abi.Elem), C.c_uint32,
                              C.POINTER(abi.Buffers), C.c_uint32, C.c_uint32, C.c_double,
                              C.POINTER(C.c_uint32), C.POINTER(abi.Stats)]
        L.wo_solve_f64.argtypes = [C.POINTER(abi.WorldDesc), C.POINTER(abi.Params), C.POINTER(abi.Elem), C.c_uint32,
                                   C.POINTER(abi.Buffers), C.c_double, C.c_uint32, C.c_void_p,
                                   C.POINTER(C.c_double)]
        L.wo_solve_f64_mg.argtypes = L.wo_solve_f64.argtypes
        L.wo_true_residual.argtypes = [C.POINTER(abi.WorldDesc), C.POINTER(abi.Params), C.POINTER(abi.Elem),
                                       C.c_uint32, C.POINTER(abi.Buffers), C.c_void_p]
        L.wo_true_residual.restype = C.c_double
        L.wo_sincos.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.wo_bind_bodies.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.wo_exact_parts.argtypes = [C.c_float, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.wo_exact_value.argtypes = [C.c_uint32, C.c_uint32]
        L.wo_exact_value.restype = C.c_float
        _lib = L
    return _lib


def _buffers(world):
    b = abi.Buffers()
    for k in abi.BUFFER_NAMES:
        arr = getattr(world, k)
        assert arr.flags["C_CONTIGUOUS"]
        setattr(b, k, arr.ctypes.data)
    return b


class Oracle:
    """Runs the oracle's passes and steps over a World's host buffers in place."""

    def __init__(self, world, elems, bodies=None):
        """bodies: a world.Bodies whose table and push sums the passes read
        and write in place (None: no free bodies)."""
        self.world = world
        self.elems = elems
        self.bodies = bodies
        self.shifted = C.c_uint32(0)

    def _bind(self):
        if self.bodies is None:
            lib().wo_bind_bodies(None, None, None)
        else:
            b = self.bodies
            assert b.motion.flags["C_CONTIGUOUS"] and b.pushes.flags["C_CONTIGUOUS"] and b.stamps.flags["C_CONTIGUOUS"]
            lib().wo_bind_bodies(b.motion.ctypes.data, b.pushes.ctypes.data, b.stamps.ctypes.data)

    def pass_(self, P, name, level=0, cycle=0):
        d = self.world.desc()
        b = _buffers(self.world)
        self._bind()
        try:
            rc = lib().wo_pass(C.byref(d), C.byref(P), self.elems, len(self.elems), C.byref(b), abi.PASS[name],
                               level, cycle)
        finally:
            lib().wo_bind_bodies(None, None, None)
        assert rc == 0, rc

    def step(self, P, max_cycles=abi.FLUID_CYCLES, flags=0, tolerance=1e-6):
        d = self.world.desc()
        b = _buffers(self.world)
        st = abi.Stats()
        self._bind()
        try:
            rc = lib().wo_step(C.byref(d), C.byref(P), self.elems, len(self.elems), C.byref(b), max_cycles, flags,
                               tolerance, C.byref(self.shifted), C.byref(st))
        finally:
            lib().wo_bind_bodies(None, None, None)
        assert rc == 0, rc
        return st

    def solve_f64(self, P, rel_tol=1e-12, max_iter=100000, multigrid=False):
        """The FP64 solve of the step's pressure system (the world stopped
        after cgAnchor): (x per cell, iterations, relative residual).
        multigrid: flexible CG preconditioned by one of the oracle's V-cycles
        (tens of iterations; leaves the V-cycle's scratch in the buffers),
        else Jacobi-preconditioned CG."""
        d = self.world.desc()
        b = _buffers(self.world)
        x = np.zeros(self.world.C, dtype=np.float64)
        rel = C.c_double(0.0)
        f = lib().wo_solve_f64_mg if multigrid else lib().wo_solve_f64
        self._bind()
        try:
            it = f(C.byref(d), C.byref(P), self.elems, len(self.elems), C.byref(b), rel_tol, max_iter,
                   x.ctypes.data, C.byref(rel))
        finally:
            lib().wo_bind_bodies(None, None, None)
        return x, it, rel.value

    def true_residual(self, P, x):
        d = self.world.desc()
        b = _buffers(self.world)
        x = np.ascontiguousarray(x, dtype=np.float32)
        self._bind()
        try:
            return lib().wo_true_residual(C.byref(d), C.byref(P), self.elems, len(self.elems), C.byref(b),
                                          x.ctypes.data)
        finally:
            lib().wo_bind_bodies(None, None, None)


def sincos(a):
    s, c = C.c_float(), C.c_float()
    lib().wo_sincos(C.c_float(a), C.byref(s), C.byref(c))
    return s.value, c.value


def exact_parts(x):
    """The oracle's exactParts of x at the push sums' scale: (low, high)."""
    lo, hi = C.c_uint32(), C.c_uint32()
    lib().wo_exact_parts(C.c_float(x), C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def exact_value(lo, hi):
    return lib().wo_exact_value(lo, hi)
