"""The C ABI's library without a GPU: it loads, exports what
include/*.h declare, agrees on layouts with the oracle and the Python
mirror, and refuses work without a device."""
import ctypes as C
import os
import re

import pytest

from worldinagrain_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include"))) if h.endswith(".h")]


def _lib():
    from worldinagrain_b200 import fluid
    return fluid.lib()


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^\s*[a-z_][a-z0-9_ \*]*?\b(wig_[a-z0-9_]+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert "wig_fluid_step" in names and "wig_fluid_residual_norm2_noalloc" in names
    assert "wig_batch_step" in names and "wig_batch_create" in names
    L = _lib()
    for n in names:
        assert hasattr(L, n), n


def test_struct_sizes():
    assert C.sizeof(abi.Params) == 80
    assert C.sizeof(abi.Elem) == 80
    assert C.sizeof(abi.Buffers) == 7 * 8
    assert C.sizeof(abi.Stats) == 9 * 4 + 3 * 4 + 3 * 8


@pytest.mark.parametrize("wh", [(1, 1), (7, 5), (64, 64), (131, 97), (256, 256), (1024, 1024), (2048, 2048), (1000, 300)])
def test_layouts_agree(wh):
    from oracle.oracle import lib as olib
    L = _lib()
    d = abi.WorldDesc(wh[0], wh[1], 0, 0)
    a, b = abi.WorldLayout(), abi.WorldLayout()
    assert L.wig_fluid_layout(C.byref(d), C.byref(a)) == 0
    assert olib().wo_layout(C.byref(d), C.byref(b)) == 0
    py = abi.layout_py(*wh)
    for f, _ in abi.WorldLayout._fields_:
        va, vb = getattr(a, f), getattr(b, f)
        if f in ("level_w", "level_h"):
            va, vb = list(va), list(vb)
        assert va == vb, f
    for k in ("capacity", "cell_count", "face_count", "block_count", "cells_bytes", "particles_bytes",
              "counters_bytes", "field_bytes", "blocks_bytes", "cg_bytes"):
        assert py[k] == getattr(a, k), k
    assert a.levels == len(py["levels"])
    lw, lh = py["levels"][-1]
    assert lw * lh <= abi.MG_COARSEST


def test_layout_rejects_bad_sizes():
    L = _lib()
    out = abi.WorldLayout()
    for w, h in ((0, 5), (5, 0), (40000, 4)):
        d = abi.WorldDesc(w, h, 0, 0)
        assert L.wig_fluid_layout(C.byref(d), C.byref(out)) == -1
        assert L.wig_fluid_last_error()


def test_create_without_a_device_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from worldinagrain_b200 import fluid
    from worldinagrain_b200 import world as W
    w = W.small_world(16, 16)
    with pytest.raises(fluid.WigError):
        fluid.LiquidStep(w, W.element_table())


def test_missing_library_raises():
    from worldinagrain_b200 import fluid
    saved = fluid._lib
    try:
        fluid._lib = None
        with pytest.raises(fluid.WigError):
            fluid.lib("/nonexistent/libwig_fluid.so")
    finally:
        fluid._lib = saved


def test_noalloc_refuses_large_worlds_without_touching_the_device():
    L = _lib()
    f = L.wig_fluid_residual_norm2_noalloc
    f.argtypes = [C.POINTER(abi.WorldDesc), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    d = abi.WorldDesc(2048, 2048, 4, 0)
    one = C.c_void_p(16)
    assert f(C.byref(d), one, one, one, one, None) == -1
    assert b"at most 16384" in L.wig_fluid_last_error()


def _header_macros():
    """The integer #defines of include/*.h, evaluated in order (a macro may
    name the ones before it)."""
    vals = {}
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        text = text.replace("\\\n", " ")
        for name, expr in re.findall(r"^#define\s+(WIG_[A-Z0-9_]+)\s+(.+)$", text, flags=re.M):
            e = re.sub(r"\b(0x[0-9a-fA-F]+|\d+)u\b", r"\1", expr.strip())
            e = re.sub(r"(\d\.\d*)f\b", r"\1", e)
            e = re.sub(r"\b(WIG_[A-Z0-9_]+)\b", lambda m: str(vals.get(m.group(1), "None")), e)
            try:
                vals[name] = eval(e, {"__builtins__": {}})
            except Exception:
                pass
    return vals


def test_body_layout_constants_agree_with_the_header():
    """The free bodies' layout constants of the Python mirror are the
    header's (js/shared.js:294-333)."""
    m = _header_macros()
    assert m["WIG_MAX_BODIES"] == abi.MAX_BODIES
    assert m["WIG_BODY_TABLE_WORDS"] == abi.BODY_TABLE_WORDS
    assert m["WIG_BODY_PUSH_WORDS"] == abi.BODY_PUSH_WORDS
    assert m["WIG_BODY_MOTION_WORDS"] == abi.BODY_MOTION_WORDS
    assert m["WIG_BODY_LIQUID_BASE"] == abi.BODY_LIQUID_BASE
    assert m["WIG_RIGID_FIX"] == abi.RIGID_FIX
    assert m["WIG_FL_LOOSE"] == abi.FL_LOOSE and m["WIG_NO_ELEM"] == abi.NO_ELEM
    assert (m["WIG_BF_ALIVE"], m["WIG_BF_NEW"], m["WIG_BF_HELD"], m["WIG_BF_WET"]) == (
        abi.BF_ALIVE, abi.BF_NEW, abi.BF_HELD, abi.BF_WET)
    for k, v in abi.BW.items():
        assert m[f"WIG_BW_{k}"] == v, k
    assert (m["WIG_BODY_TILE"], m["WIG_BODY_STAT_WORDS"], m["WIG_BODY_COUNTERS"], m["WIG_BODY_SUM_WORDS"]) == (
        abi.BODY_TILE, abi.BODY_STAT_WORDS, abi.BODY_COUNTERS, abi.BODY_SUM_WORDS)
    assert m["WIG_CLAIM_PERIOD"] == abi.CLAIM_PERIOD
