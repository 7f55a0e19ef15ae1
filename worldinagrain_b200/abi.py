"""ctypes mirror of include/wig_fluid.h (structs, constants, pass ids).

The C header is the boundary; this module only restates its types for the
Python host side and the tests.
"""
import ctypes as C

ABI_VERSION = 2

FLUID_BLOCK = 8
LIQUID_CELL_WORDS = 11
MG_COARSEST = 512
MG_LEVELS = 8
FLUID_STATS = 9
FLUID_CYCLES = 16

COUNT_ACTIVE, COUNT_RETIRED, COUNT_VISCOUS, COUNT_PARTICLES = 0, 1, 2, 3
COUNT_RESIDUAL, COUNT_CYCLES, COUNT_MOST_CYCLES = 4, 7, 8

KIND_SOLID, KIND_POWDER, KIND_LIQUID, KIND_GAS = 1, 2, 3, 4
AIR, WALL, SAND, WATER = 0, 1, 2, 3
NO_ELEM = 255
FL_LOOSE = 8

# Free bodies (include/wig_fluid.h, js/shared.js:294-333)
MAX_BODIES = 1024
BODY_TABLE_WORDS = 116
BODY_CONTACTS = 16384
BODY_CONTACT_WORDS = 12
BODY_LIQUID_WORDS = 4
BODY_PUSH_WORDS = 36
BODY_LIQUID_BASE = MAX_BODIES * (1 + BODY_TABLE_WORDS) + BODY_CONTACTS * BODY_CONTACT_WORDS
BODY_MOTION_WORDS = BODY_LIQUID_BASE + MAX_BODIES * BODY_LIQUID_WORDS
BW = dict(POS=0, VEL=3, SPIN=5, MASS=6, INERTIA=7, CELLS=13, FLAGS=18, FRAME=19, SUBCELL=25, CARGO=105, CARGO_INERTIA=106,
          MOBILITY=108, MOBILITY_AT=114)
BF_ALIVE, BF_NEW, BF_HELD, BF_WET = 1, 2, 32, 64
RIGID_FIX = 16777216.0
BODY_TILE, BODY_STAT_WORDS, BODY_COUNTERS, BODY_SUM_WORDS = 8, 8, 9, 8
CLAIM_PERIOD = 0xfffff


def body_stamps_layout(width, height):
    """(words of the bodies' buffer, first swept-stamp word) of a world
    (js/sim.js:796-799, shaders/common.wgsl:316-380): cell i's stamp of step
    f is at first + 2 i + (f & 1)."""
    tiles = -(-width // BODY_TILE) * -(-height // BODY_TILE)
    n = width * height
    header = 4 * tiles + BODY_STAT_WORDS + BODY_COUNTERS + MAX_BODIES
    first = header + (2 + BODY_SUM_WORDS) * n + 1 + tiles + 2 * n + n
    return header + (2 + BODY_SUM_WORDS) * n + 1 + tiles + 5 * n, first

WIG_OK = 0
ERRORS = {
    -1: "WIG_E_ARG", -2: "WIG_E_OOM", -3: "WIG_E_CUDA", -4: "WIG_E_CAPACITY",
    -5: "WIG_E_NOT_CONVERGED", -6: "WIG_E_STATE", -7: "WIG_E_NO_DEVICE",
}

STEP_BOOKKEEPING_ONLY = 1
STEP_SHIFTED_SET = 2
STEP_SHIFTED_FIRST = 4
STEP_VISCOUS = 8
STEP_TOLERANCE = 16
STEP_F64_DOTS = 32
STEP_SYNC_STATS = 64
STEP_PLAIN = 128
STEP_PERSISTENT = 256
STEP_MIXED = 512

# wig_launch_knob (include/wig_batch.h): launch shapes that change no result
LAUNCH_COARSE_CELLS = 0
LAUNCH_LEVEL_PER_SM = 1
LAUNCH_CG_PER_SM = 2
LAUNCH_RELAX_PER_SM = 3
LAUNCH_KNOBS = {"coarse_cells": LAUNCH_COARSE_CELLS, "level_per_sm": LAUNCH_LEVEL_PER_SM,
                "cg_per_sm": LAUNCH_CG_PER_SM, "relax_per_sm": LAUNCH_RELAX_PER_SM}

PASSES = [
    "SYNC", "SYNC_MARKS", "SYNC_PARTICLES", "SYNC_SEED", "COMPACT", "RETIRE", "CLEAR", "GATHER",
    "SEAL_JOIN", "SEAL_ANCHOR", "CLASSIFY", "SET_FACES", "VISCOSITY_RED", "VISCOSITY_BLACK", "UNPRESS",
    "DIVERGENCE", "CG_START", "CG_JOIN", "CG_ANCHOR", "CG_RESIDUAL", "CG_PREPARE", "RELAX_RIMS", "RELAX",
    "RELAX_SHIFTED", "RESTRICT", "SMOOTH_RED", "SMOOTH_BLACK", "SOLVE", "PROLONG", "PROLONG_FINE",
    "CG_RHO", "CG_BETA", "CG_DIRECTION", "CG_APPLY", "CG_ALPHA", "CG_UPDATE", "CG_FINISH", "PROJECT",
    "EXTRAPOLATE", "EXTRAPOLATE_FURTHER", "ADVECT", "SORT_COUNT", "SCAN_BLOCKS", "SCAN_TOTALS",
    "SCAN_FINISH", "SCATTER", "RASTER_CLAIMS", "RASTER", "UNPAINT",
    "BODY_START", "BODY_LOADS", "BODY_DRAG", "BODY_FACES", "CG_BODY_X", "CG_BODY_P", "CG_BODY_F",
    "RIGIDIFY", "BODY_PUSH",
]
PASS = {name: i for i, name in enumerate(PASSES)}
PROFILE_NAMES = PASSES + ["NORM", "REPORT", "F_SETUP", "F_LOOP", "F_RELAX", "F_RESTRICT", "F_SMOOTH", "F_COARSE",
                          "F_PROLONG", "F_PROLONG_FINE", "F_RHO_BETA", "F_DIRECTION", "F_APPLY_ALPHA", "F_UPDATE",
                          "F_FINISH", "F_SOLVE", "SCHED"]
PROFILE_SLOTS = len(PROFILE_NAMES)


class Params(C.Structure):
    """Params (shaders/common.wgsl:5-40), 80 bytes."""
    _fields_ = [
        ("size", C.c_uint32 * 2), ("frame", C.c_uint32), ("seed", C.c_uint32),
        ("offset", C.c_uint32 * 2), ("support_max", C.c_float), ("dx", C.c_float),
        ("day", C.c_float), ("day_rate", C.c_float), ("hole_pull", C.c_float),
        ("mass_pull", C.c_float), ("earth_g", C.c_float), ("dt", C.c_float),
        ("day_dt", C.c_float), ("clock_span", C.c_float), ("heat_stages", C.c_uint32),
        ("heat_limit", C.c_float), ("holding", C.c_uint32), ("pad", C.c_float),
    ]


class Elem(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32), ("density", C.c_float), ("weight", C.c_float), ("heat_cap", C.c_float),
        ("viscosity", C.c_float), ("viscosity_t", C.c_float), ("viscosity_e", C.c_float),
        ("tension", C.c_float), ("expansion", C.c_float), ("expansion2", C.c_float),
        ("hi_t", C.c_float), ("lo_t", C.c_float), ("up_span", C.c_float), ("down_span", C.c_float),
        ("down_scale", C.c_float), ("sol_density", C.c_float), ("flags", C.c_uint32),
        ("wetting", C.c_float), ("break_to", C.c_uint32), ("pad", C.c_float),
    ]


class WorldDesc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32),
                ("liquid_per_cell", C.c_uint32), ("capacity", C.c_uint32)]


class WorldLayout(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("liquid_per_cell", C.c_uint32),
        ("capacity", C.c_uint32), ("cell_count", C.c_uint32), ("face_count", C.c_uint32),
        ("block_count", C.c_uint32), ("blocks_wide", C.c_uint32), ("edge_tiles", C.c_uint32),
        ("levels", C.c_uint32), ("level_w", C.c_uint32 * MG_LEVELS), ("level_h", C.c_uint32 * MG_LEVELS),
        ("cells_bytes", C.c_uint64), ("particles_bytes", C.c_uint64), ("counters_bytes", C.c_uint64),
        ("field_bytes", C.c_uint64), ("blocks_bytes", C.c_uint64), ("cg_bytes", C.c_uint64),
    ]


class Buffers(C.Structure):
    _fields_ = [("cells", C.c_void_p), ("sorted", C.c_void_p), ("parts", C.c_void_p),
                ("counters", C.c_void_p), ("field", C.c_void_p), ("blocks", C.c_void_p),
                ("cg", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("count", C.c_uint32 * FLUID_STATS), ("particles", C.c_uint32), ("cycles", C.c_uint32),
                ("launches", C.c_uint32), ("rel_residual", C.c_double), ("b_norm", C.c_double),
                ("true_residual", C.c_double)]


BUFFER_NAMES = ("cells", "sorted", "parts", "counters", "field", "blocks", "cg")


def layout_py(width, height, liquid_per_cell=4, capacity=0):
    """The reference's sizes for a world (js/sim.js:741-843), computed in Python."""
    import math
    W, H = int(width), int(height)
    C_ = W * H
    F = (W + 1) * H + W * (H + 1)
    ppc = liquid_per_cell or 4
    cap = capacity or math.ceil(C_ * ppc * 1.25)
    bw = (W + 7) // 8
    B = bw * ((H + 7) // 8)
    levels = []
    for l in range(1, MG_LEVELS + 1):
        lw, lh = (W + (1 << l) - 1) >> l, (H + (1 << l) - 1) >> l
        levels.append((lw, lh))
        if lw * lh <= MG_COARSEST:
            break
    level_cells = sum(a * b for a, b in levels)
    return {
        "width": W, "height": H, "liquid_per_cell": ppc, "capacity": cap, "cell_count": C_,
        "face_count": F, "block_count": B, "blocks_wide": bw, "edge_tiles": bw + (H + 7) // 8 + 1,
        "levels": levels,
        "cells_bytes": 16 * (C_ + (C_ + 1) // 2),
        "particles_bytes": 16 + 48 * cap,
        "counters_bytes": 4 * (11 * C_ + 2 * F),
        "field_bytes": 16 * ((C_ + level_cells) * 2 + F + 2 * ((F + 3) // 4)),
        "blocks_bytes": 4 * (5 * B + FLUID_STATS),
        "cg_bytes": 16 * (C_ + B + 1),
    }
