/*
 * wig_fluid.h — C ABI of the B200 liquid step (worldinagrain_b200).
 *
 * This library is a drop-in for the liquid passes that the reference's
 * `Simulation.encodeFluid(pass, offset)` (js/sim.js:2466-2612) records into a
 * WebGPU compute pass.  The reference binds one group of 17 bindings
 * (js/sim.js:407-410, js/sim.js:1155-1159, shaders/fluid.wgsl:116-181,
 * :2543, :2547); this header takes the same buffers as plain device pointers
 * in the same layouts, so a host that owns the reference's buffers can hand
 * them over unchanged:
 *
 *   binding 0  Params        -> wig_params (host struct, copied per step)
 *   binding 1  elems         -> wig_elem table (the liquid's fields only)
 *   binding 2  cells         -> cells      (vec4<u32> per cell, then gas plane)
 *   binding 3  air           -> (not bound: the configs carry no air motion)
 *   binding 4  sorted        -> sorted     (Particles: 16 B header + 3 planes)
 *   binding 5  parts         -> parts      (Particles)
 *   binding 6  counters      -> counters   (u32: 11 per cell, 2 per face)
 *   binding 7  field         -> field      (vec4<f32>: 2 per cell, faces, levels)
 *   binding 8  blocks        -> blocks     (u32: 5 per 8x8 block + 9 stats)
 *   binding 9  Level         -> (level, cycle) arguments of wig_fluid_dispatch
 *   binding 10 gravity       -> (not bound: Earth's pull P.earthG straight down)
 *   binding 11 airSource     -> (not bound)
 *   binding 12 bodyMotion    -> motion     (u32: the body table, wig_fluid_bind_bodies; optional)
 *   binding 13 occupants     -> (not bound: no people)
 *   binding 14 bodies        -> stamps     (u32: the bodies' buffer, read for its swept stamps; optional)
 *   binding 15 fluidCg       -> cg         (vec4<f32>: per cell, per block, sums)
 *   binding 16 bodyPushes    -> pushes     (u32: WIG_BODY_PUSH_WORDS per body; optional)
 *
 * All entry points return 0 on success and a negative WIG_E* code on error;
 * wig_fluid_last_error() gives a one-line description of the last error on
 * the calling thread.  No C++ exception crosses this boundary.  A handle is
 * not thread-safe and works on the one CUDA stream passed to it.
 */
#ifndef WIG_FLUID_H
#define WIG_FLUID_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WIG_ABI_VERSION 2u

/* Error codes. */
#define WIG_OK 0
#define WIG_E_ARG (-1)        /* bad argument or descriptor */
#define WIG_E_OOM (-2)        /* device allocation failed */
#define WIG_E_CUDA (-3)       /* a CUDA call failed (message names it) */
#define WIG_E_CAPACITY (-4)   /* more particles than the buffers hold */
#define WIG_E_NOT_CONVERGED (-5) /* solve left more than the tolerance after max_cycles */
#define WIG_E_STATE (-6)      /* call out of order (e.g. step before bind) */
#define WIG_E_NO_DEVICE (-7)  /* no CUDA device usable */

/* Layout constants shared with the reference (js/shared.js:263-282). */
#define WIG_FLUID_BLOCK 8u
#define WIG_LIQUID_CELL_WORDS 11u
#define WIG_MG_COARSEST 512u
#define WIG_MG_LEVELS 8u
#define WIG_FLUID_STATS 9u
#define WIG_FLUID_CYCLES 16u
#define WIG_PARTICLES_HEADER 16u
#define WIG_PARTICLE_BYTES 48u

/* FLUID_COUNT word offsets (js/shared.js:271). */
#define WIG_COUNT_ACTIVE 0u
#define WIG_COUNT_RETIRED 1u
#define WIG_COUNT_VISCOUS 2u
#define WIG_COUNT_PARTICLES 3u
#define WIG_COUNT_RESIDUAL 4u
#define WIG_COUNT_CYCLES 7u
#define WIG_COUNT_MOST_CYCLES 8u

/* Element kinds (js/elements.js:8). */
#define WIG_KIND_SOLID 1u
#define WIG_KIND_POWDER 2u
#define WIG_KIND_LIQUID 3u
#define WIG_KIND_GAS 4u

/* Element ids the liquid step names itself (js/elements.js DEFS order). */
#define WIG_ELEM_AIR 0u
#define WIG_ELEM_WALL 1u
#define WIG_ELEM_SAND 2u
#define WIG_ELEM_WATER 3u
#define WIG_MAX_ELEMS 256u
#define WIG_NO_ELEM 255u      /* js/shared.js:113 */
#define WIG_FL_LOOSE 8u       /* a cell's flag: moving with a free body (shaders/common.wgsl:160) */

/* Free bodies (js/shared.js:294-333).  The body table `motion` (binding 12)
 * holds MAX_BODIES list words, then MAX_BODIES slots of BODY_TABLE_WORDS
 * (word WIG_BW_* of body b at MAX_BODIES + b * BODY_TABLE_WORDS + k), the
 * contacts, and BODY_LIQUID_WORDS a body of what the liquid did to it this
 * step (velocity x, y and spin in RIGID_FIX fixed point, and LIQUID_WET).
 * `pushes` (binding 16) is the solve's scratch: BODY_PUSH_SETS sets a body
 * of a force x, y and a torque, each an exact sum in two words. */
#define WIG_MAX_BODIES 1024u
#define WIG_BODY_TABLE_WORDS 116u
#define WIG_BODY_CONTACTS 16384u
#define WIG_BODY_CONTACT_WORDS 12u
#define WIG_BODY_LIQUID_WORDS 4u
#define WIG_BODY_PUSH_SETS 6u
#define WIG_BODY_PUSH_WORDS (6u * WIG_BODY_PUSH_SETS)
#define WIG_BODY_MOTION_WORDS (WIG_MAX_BODIES * (1u + WIG_BODY_TABLE_WORDS) + \
                               WIG_BODY_CONTACTS * WIG_BODY_CONTACT_WORDS + WIG_MAX_BODIES * WIG_BODY_LIQUID_WORDS)
#define WIG_BODY_LIQUID_BASE (WIG_MAX_BODIES * (1u + WIG_BODY_TABLE_WORDS) + WIG_BODY_CONTACTS * WIG_BODY_CONTACT_WORDS)
#define WIG_BW_POS 0u            /* vec2 f32: the centre of mass, cells */
#define WIG_BW_VEL 3u            /* vec2 f32: cells/step */
#define WIG_BW_SPIN 5u           /* f32: radians/step */
#define WIG_BW_MASS 6u
#define WIG_BW_INERTIA 7u
#define WIG_BW_CELLS 13u         /* u32 */
#define WIG_BW_FLAGS 18u         /* u32: WIG_BF_* */
#define WIG_BW_FRAME 19u         /* u32: the step the body was last stamped */
#define WIG_BW_SUBCELL 25u       /* 2 x f16: the pose's offset from the stamp, cells */
#define WIG_BW_CARGO 105u
#define WIG_BW_CARGO_INERTIA 106u
#define WIG_BW_MOBILITY 108u     /* 6 f32: a symmetric 3 x 3 (the contacts' give) */
#define WIG_BW_MOBILITY_AT 114u  /* u32: the step MOBILITY was worked out */
#define WIG_BF_ALIVE 1u
#define WIG_BF_NEW 2u
#define WIG_BF_HELD 32u
#define WIG_BF_WET 64u
#define WIG_RIGID_FIX 16777216.0f
/* The bodies' buffer (binding 14, js/sim.js:796-799) of a W x H world: its
 * header (4 T + BODY_STAT_WORDS + BODY_COUNTERS + MAX_BODIES words, T the
 * 8 x 8 body tiles), 2 + BODY_SUM_WORDS words a cell, structure's words
 * (1 + T + 2 W H), and per cell two swept stamps, one for even steps and one
 * for odd (shaders/common.wgsl:316-380): which body last moved over the cell
 * as its cup (bit 0 clear) or a seam of its wall (bit 0 set), the stamp's
 * step in the top 20 bits. */
#define WIG_BODY_TILE 8u
#define WIG_BODY_STAT_WORDS 8u
#define WIG_BODY_COUNTERS 9u
#define WIG_BODY_SUM_WORDS 8u
#define WIG_CLAIM_PERIOD 0xfffffu
#define WIG_LIQUID_WET 0x80000000u

/* Params (shaders/common.wgsl:5-40), 80 bytes, written per step by the host
 * (js/sim.js:1975-1995).  Field for field the reference's uniform. */
typedef struct wig_params {
    uint32_t size[2];
    uint32_t frame;
    uint32_t seed;
    uint32_t offset[2];
    float support_max;
    float dx;
    float day;
    float day_rate;
    float hole_pull;
    float mass_pull;
    float earth_g;   /* cells/step^2, straight down the screen (+y) */
    float dt;
    float day_dt;
    float clock_span;
    uint32_t heat_stages;
    float heat_limit;
    uint32_t holding;
    float pad;
} wig_params;

/* The fields of the reference's Elem (js/elements.js:44-300) that the liquid
 * step reads, one 80-byte record per element id. */
typedef struct wig_elem {
    uint32_t kind;
    float density;      /* g/cm^3 x 100, water 100 */
    float weight;       /* cells/step^2 */
    float heat_cap;
    float viscosity;
    float viscosity_t;
    float viscosity_e;
    float tension;
    float expansion;
    float expansion2;
    float hi_t;
    float lo_t;
    float up_span;
    float down_span;
    float down_scale;
    float sol_density;
    uint32_t flags;     /* F_* (js/elements.js:10-21); F_IMPACT = 32 */
    float wetting;
    uint32_t break_to;  /* breakTo (js/elements.js:160): WIG_NO_ELEM for none; a loose solid
                           with one is a free body's cell (fluid.wgsl:1233-1248) */
    float pad;
} wig_elem;

/* A world: its size and the liquid's particles per cell (LIQUID_PER_CELL,
 * js/shared.js:276; 4 in the reference, a parameter here). */
typedef struct wig_world_desc {
    uint32_t width;
    uint32_t height;
    uint32_t liquid_per_cell;   /* 0 means the reference's 4 */
    uint32_t capacity;          /* particle slots; 0 means ceil(W*H*ppc*1.25) */
} wig_world_desc;

/* Sizes (bytes) and shape the reference derives for a world
 * (js/sim.js:741-843). */
typedef struct wig_world_layout {
    uint32_t width, height, liquid_per_cell, capacity;
    uint32_t cell_count, face_count, block_count, blocks_wide, edge_tiles;
    uint32_t levels;                 /* coarse levels (js/sim.js:763-771) */
    uint32_t level_w[WIG_MG_LEVELS];
    uint32_t level_h[WIG_MG_LEVELS];
    uint64_t cells_bytes;            /* C vec4 + ceil(C/2) vec4 gas plane */
    uint64_t particles_bytes;        /* 16 + 48 * capacity */
    uint64_t counters_bytes;         /* (11 C + 2 F) * 4 */
    uint64_t field_bytes;            /* ((C + level cells) * 2 + F + 2 ceil(F/4)) * 16 */
    uint64_t blocks_bytes;           /* (5 B + 9) * 4 */
    uint64_t cg_bytes;               /* (C + B + 1) * 16 */
} wig_world_layout;

/* Device pointers for the bound buffers (layouts as in the comment above).
 * A null pointer asks the handle to allocate that buffer itself. */
typedef struct wig_fluid_buffers {
    void* cells;
    void* sorted;
    void* parts;
    void* counters;
    void* field;
    void* blocks;
    void* cg;
} wig_fluid_buffers;

/* Step flags. */
#define WIG_STEP_BOOKKEEPING_ONLY 1u  /* fluidStats.active == 0: syncMarks, compact, retire */
#define WIG_STEP_SHIFTED_SET 2u       /* take the tiling parity from the next bit */
#define WIG_STEP_SHIFTED_FIRST 4u     /* (with SHIFTED_SET) the step's first relaxation is shifted */
#define WIG_STEP_VISCOUS 8u           /* encode viscosity sweeps (fluidStats.viscous) */
#define WIG_STEP_TOLERANCE 16u        /* stop on ||r||2/||b||2 <= tol (FP64) instead of max|r| < 1e-2 */
#define WIG_STEP_F64_DOTS 32u         /* CG dot products in FP64 */
#define WIG_STEP_SYNC_STATS 64u       /* copy the stats to the host at the end of the step */
#define WIG_STEP_PLAIN 128u           /* the solve as one kernel per reference pass (else the fast form) */
#define WIG_STEP_PERSISTENT 256u      /* the fast form's iterations as one persistent cooperative kernel (else kernels in a graph WHILE loop) */
#define WIG_STEP_MIXED 512u           /* mixed precision (fast form, with TOLERANCE and F64_DOTS): the multigrid levels
                                         stored in 16 bits and worked in FP32 (each coarse level's density and stencil
                                         coefficients in binary16, its potentials, right-hand sides and way-up potentials
                                         in bf16; the fine smoother's coefficients in binary16 copies), the fine level's
                                         potentials and the CG vectors and operator FP32, dots and norms FP64; every 8th
                                         iteration and before the solve stops, the true residual b + A x worked in FP64
                                         and put in for the recursive one when it has drifted above it and above the
                                         FP32 rounding floor of A x; not bit-exact with the other forms */

/* Per-step statistics (the report words, js/sim.js:1882-1900, plus the
 * solve's residuals). */
typedef struct wig_fluid_stats {
    uint32_t count[WIG_FLUID_STATS];  /* FLUID_COUNT words */
    uint32_t particles;               /* sorted.count after the step */
    uint32_t cycles;                  /* CG iterations run this step */
    uint32_t launches;                /* kernels the last step launched */
    double rel_residual;              /* ||r||2/||b||2 of the CG (recursive) residual, FP64 (tolerance mode) */
    double b_norm;                    /* ||b||2 at the solve's start */
    double true_residual;             /* the mixed form: ||b + A x||2/||b||2 worked in FP64 at its last check (else 0) */
} wig_fluid_stats;

typedef struct wig_fluid wig_fluid;

/* Pass ids, one per reference pipeline dispatched by encodeFluid. */
enum wig_pass {
    WIG_PASS_SYNC = 0,            /* fluid.wgsl:637 */
    WIG_PASS_SYNC_MARKS,          /* fluid.wgsl:652 */
    WIG_PASS_SYNC_PARTICLES,      /* fluid.wgsl:767 */
    WIG_PASS_SYNC_SEED,           /* fluid.wgsl:863 */
    WIG_PASS_COMPACT,             /* fluid.wgsl:896 */
    WIG_PASS_RETIRE,              /* fluid.wgsl:924 */
    WIG_PASS_CLEAR,               /* fluid.wgsl:962 */
    WIG_PASS_GATHER,              /* fluid.wgsl:1017 */
    WIG_PASS_SEAL_JOIN,           /* fluid.wgsl:1531 */
    WIG_PASS_SEAL_ANCHOR,         /* fluid.wgsl:1545 */
    WIG_PASS_CLASSIFY,            /* fluid.wgsl:1578 */
    WIG_PASS_SET_FACES,           /* fluid.wgsl:1982 */
    WIG_PASS_VISCOSITY_RED,       /* fluid.wgsl:3458 */
    WIG_PASS_VISCOSITY_BLACK,     /* fluid.wgsl:3463 */
    WIG_PASS_UNPRESS,             /* fluid.wgsl:3453 */
    WIG_PASS_DIVERGENCE,          /* fluid.wgsl:1996 */
    WIG_PASS_CG_START,            /* fluid.wgsl:2665 */
    WIG_PASS_CG_JOIN,             /* fluid.wgsl:2677 */
    WIG_PASS_CG_ANCHOR,           /* fluid.wgsl:2692 */
    WIG_PASS_CG_RESIDUAL,         /* fluid.wgsl:2708 */
    WIG_PASS_CG_PREPARE,          /* fluid.wgsl:2721 */
    WIG_PASS_RELAX_RIMS,          /* fluid.wgsl:2096 */
    WIG_PASS_RELAX,               /* fluid.wgsl:2184 */
    WIG_PASS_RELAX_SHIFTED,       /* fluid.wgsl:2189 */
    WIG_PASS_RESTRICT,            /* fluid.wgsl:2342 */
    WIG_PASS_SMOOTH_RED,          /* fluid.wgsl:2379 */
    WIG_PASS_SMOOTH_BLACK,        /* fluid.wgsl:2384 */
    WIG_PASS_SOLVE,               /* fluid.wgsl:2407 */
    WIG_PASS_PROLONG,             /* fluid.wgsl:2459 */
    WIG_PASS_PROLONG_FINE,        /* fluid.wgsl:2500 */
    WIG_PASS_CG_RHO,              /* fluid.wgsl:2736 */
    WIG_PASS_CG_BETA,             /* fluid.wgsl:2752 */
    WIG_PASS_CG_DIRECTION,        /* fluid.wgsl:2767 */
    WIG_PASS_CG_APPLY,            /* fluid.wgsl:2779 */
    WIG_PASS_CG_ALPHA,            /* fluid.wgsl:2797 */
    WIG_PASS_CG_UPDATE,           /* fluid.wgsl:2852 */
    WIG_PASS_CG_FINISH,           /* fluid.wgsl:2884 */
    WIG_PASS_PROJECT,             /* fluid.wgsl:2925 */
    WIG_PASS_EXTRAPOLATE,         /* fluid.wgsl:3267 */
    WIG_PASS_EXTRAPOLATE_FURTHER, /* fluid.wgsl:3272 */
    WIG_PASS_ADVECT,              /* fluid.wgsl:3616 */
    WIG_PASS_SORT_COUNT,          /* fluid.wgsl:3700 */
    WIG_PASS_SCAN_BLOCKS,         /* fluid.wgsl:3730 */
    WIG_PASS_SCAN_TOTALS,         /* fluid.wgsl:3757 */
    WIG_PASS_SCAN_FINISH,         /* fluid.wgsl:3783 */
    WIG_PASS_SCATTER,             /* fluid.wgsl:3793 */
    WIG_PASS_RASTER_CLAIMS,       /* fluid.wgsl:3928 */
    WIG_PASS_RASTER,              /* fluid.wgsl:3983 */
    WIG_PASS_UNPAINT,             /* fluid.wgsl:4163 */
    WIG_PASS_BODY_START,          /* fluid.wgsl:3079 */
    WIG_PASS_BODY_LOADS,          /* fluid.wgsl:3094 */
    WIG_PASS_BODY_DRAG,           /* fluid.wgsl:3149 */
    WIG_PASS_BODY_FACES,          /* fluid.wgsl:3180 */
    WIG_PASS_CG_BODY_X,           /* fluid.wgsl:2820 */
    WIG_PASS_CG_BODY_P,           /* fluid.wgsl:2828 */
    WIG_PASS_CG_BODY_F,           /* fluid.wgsl:2840 */
    WIG_PASS_RIGIDIFY,            /* fluid.wgsl:3034 */
    WIG_PASS_BODY_PUSH,           /* fluid.wgsl:3205 */
    WIG_PASS_COUNT
};

/* The layout the reference derives for a world (js/sim.js:741-843). */
int wig_fluid_layout(const wig_world_desc* d, wig_world_layout* out);

/* Replaces `new Simulation(...)`'s liquid allocations (js/sim.js:741-843):
 * creates a handle on the current CUDA device for world d with element table
 * elems[n_elems]. */
int wig_fluid_create(const wig_world_desc* d, const wig_elem* elems, uint32_t n_elems,
                     wig_fluid** out);

/* Replaces the bind group (js/sim.js:1155-1159): adopts caller-owned device
 * buffers (null fields are allocated by the handle and zeroed, as
 * js/sim.js:1259 `clear` leaves them). */
int wig_fluid_bind(wig_fluid* h, const wig_fluid_buffers* b);

/* Binds the free bodies' buffers (bindings 12, 14 and 16, js/sim.js:1159):
 * the body table `motion` (WIG_BODY_MOTION_WORDS u32, caller-owned, read for
 * the bodies' poses and written in its liquid words), `pushes`
 * (WIG_MAX_BODIES * WIG_BODY_PUSH_WORDS u32, caller-owned scratch), and
 * optionally `stamps`, the bodies' buffer (layout above, read only: the
 * swept stamps of last step and the one before, by which a body's seams
 * and cup are found; null: no body has seams or a cup).  With them bound,
 * each step couples the bodies into the solve (A = L + J^T M^-1 J,
 * fluid.wgsl:1181-1470, :2819-2845, :2949-3218) and runs in the plain form
 * (a kernel per reference pass), whatever the form flags ask.  motion and
 * pushes null unbind all three.  Single-world handles only. */
int wig_fluid_bind_bodies(wig_fluid* h, void* motion, void* pushes, void* stamps);

/* The bound (or allocated) device buffers. */
int wig_fluid_buffers_of(wig_fluid* h, wig_fluid_buffers* out);

/* Replaces encodeFluid (js/sim.js:2466-2612): one liquid step, stream
 * ordered and asynchronous on `stream` (a cudaStream_t, 0 for the legacy
 * stream).  max_cycles is fluidCycles (<= 64); flags WIG_STEP_*.
 * tolerance is used with WIG_STEP_TOLERANCE. */
int wig_fluid_step(wig_fluid* h, const wig_params* P, uint32_t max_cycles, uint32_t flags,
                   double tolerance, void* stream);

/* One reference pipeline dispatch (encodeFluid's `run`/`blocks`/`particles`
 * with its Level slot): pass id, level index and cycle. */
int wig_fluid_dispatch(wig_fluid* h, const wig_params* P, int pass, uint32_t level,
                       uint32_t cycle, void* stream);

/* Host <-> device copies of one bound buffer (which: 0 cells, 1 sorted,
 * 2 parts, 3 counters, 4 field, 5 blocks, 6 cg), stream ordered on the
 * handle's stream and complete on return: the reference's
 * device.queue.writeBuffer and mapped readbacks (js/sim.js:1259,
 * js/snapshot.js:97-164) for worlds loaded or saved by the host. */
int wig_fluid_upload(wig_fluid* h, int which, const void* host, uint64_t offset, uint64_t bytes, void* stream);
int wig_fluid_download(wig_fluid* h, int which, void* host, uint64_t offset, uint64_t bytes, void* stream);

/* Profile slots: one per pass id, then the tolerance form's norm kernel,
 * the report kernel, and the kernels of the fast form of the solve. */
enum wig_profile_slot {
    WIG_SLOT_NORM = WIG_PASS_COUNT,
    WIG_SLOT_REPORT,
    WIG_SLOT_F_SETUP,
    WIG_SLOT_F_LOOP,
    WIG_SLOT_F_RELAX,
    WIG_SLOT_F_RESTRICT,
    WIG_SLOT_F_SMOOTH,
    WIG_SLOT_F_COARSE,
    WIG_SLOT_F_PROLONG,
    WIG_SLOT_F_PROLONG_FINE,
    WIG_SLOT_F_RHO_BETA,
    WIG_SLOT_F_DIRECTION,
    WIG_SLOT_F_APPLY_ALPHA,
    WIG_SLOT_F_UPDATE,
    WIG_SLOT_F_FINISH,
    WIG_SLOT_F_SOLVE,
    WIG_SLOT_SCHED,        /* writing a batch's work lists */
    WIG_PROFILE_SLOTS
};

/* One step as wig_fluid_step, but launched pass by pass with CUDA events
 * around each launch (the reference's per-phase GPU timestamps,
 * js/timer.js:7-98): per slot, the summed milliseconds in ms_out and the
 * launches in calls_out (WIG_PROFILE_SLOTS entries each).  Synchronous. */
int wig_fluid_step_profile(wig_fluid* h, const wig_params* P, uint32_t max_cycles, uint32_t flags, double tolerance,
                           void* stream, float* ms_out, uint32_t* calls_out);

/* The fast form's launch shapes of this world (knob: enum wig_launch_knob of
 * wig_batch.h, the same values and ranges): none changes a result.  No
 * counterpart in the reference, whose dispatch sizes are fixed per pipeline
 * (encodeFluid's run and blocks, js/sim.js:2473-2478). */
int wig_fluid_set_launch(wig_fluid* h, uint32_t knob, uint32_t value);
int wig_fluid_get_launch(const wig_fluid* h, uint32_t knob, uint32_t* value);

/* Replaces readReport (js/sim.js:1882-1900): waits for the stream and reads
 * the FLUID_COUNT words and the solve's statistics of the last step.  The
 * report is filled in whatever the return code.  WIG_E_NOT_CONVERGED: the
 * step ran WIG_STEP_TOLERANCE with a nonzero right-hand side and its solve
 * stopped after max_cycles with rel_residual above the tolerance (the step
 * is complete; a host that adapts max_cycles from the report, as
 * js/sim.js:1896-1900 adapts fluidCycles, raises it).  The reference's own
 * criterion (max|r| < 1e-2, without WIG_STEP_TOLERANCE) reports no such
 * error: it stops at max_cycles as the reference does.  WIG_E_CAPACITY: the
 * step's sync and seeding put more particles into `parts` than its
 * capacity (fluid.wgsl:104-107, :827-830); those past the room are lost.
 * WIG_E_STATE (a device loop gave up at its bound) takes precedence over
 * WIG_E_CAPACITY, which takes precedence over WIG_E_NOT_CONVERGED. */
int wig_fluid_read_stats(wig_fluid* h, wig_fluid_stats* out);

void wig_fluid_destroy(wig_fluid* h);

/* No counterpart in the reference.  For hosts that own all device memory
 * and cannot let a library call cudaMalloc (work recorded into a CUDA graph
 * while it runs, one pre-reserved pool managed by the host's own allocator,
 * a real-time path): the squared FP64 norm, over the liquid cells (field's
 * z > 0) of the blocks worked on, of the pressure solve's residual r (cg's
 * y per cell), summed in the same order as wig_fluid_step's tolerance form
 * sums it (so it equals wig_fluid_stats' (rel_residual * b_norm)^2 after a
 * tolerance-form step).  The caller passes the world's shape, its field,
 * blocks and cg buffers, and a device double for the result, written on
 * `stream`.  It allocates nothing: its per-block scratch is a static device
 * array of WIG_NOALLOC_MAX_BLOCKS doubles (128 KiB held on every GPU that
 * loads the library until the process exits), so worlds of more blocks are
 * refused with WIG_E_ARG.  The first call on a device looks up that array's
 * device address; make it before any stream capture.  Calls share the one
 * array: calls whose work overlaps on the GPU race. */
#define WIG_NOALLOC_MAX_BLOCKS 16384u
int wig_fluid_residual_norm2_noalloc(const wig_world_desc* d, const void* field, const void* blocks, const void* cg,
                                     double* out, void* stream);

/* No counterpart in the reference.  The allocation-free entry point keeps
 * its array's device address per device for the process's life; a host that
 * destroys and recreates the current device's primary context
 * (cudaDeviceReset) calls this afterwards, so the next call looks the
 * address up again in the new context. */
int wig_fluid_noalloc_forget_device(void);

/* No counterpart in the reference.  Lowers the bounds of the device's
 * waits on the current device, for every kernel launched after the call
 * (graphs already captured included): loop_limit bounds each lock-free
 * retry loop (the union-find of sealJoin and cgJoin, label.wgsl:27-55),
 * spin_limit the polls of the persistent form's grid barrier.  0 restores a
 * default (2^22 retries; 2^23 polls of about 64 ns).  A loop that runs out
 * gives up, and the step's stats read returns WIG_E_STATE; nothing hangs
 * and the device stays usable.  For tests of those failure paths: a host
 * has no other reason to call it.  Limits above the defaults are refused
 * with WIG_E_ARG.  Synchronous (it writes two device words). */
int wig_fluid_set_wait_limits(uint32_t loop_limit, uint32_t spin_limit);

/* One-line description of the last error on this thread ("" if none). */
const char* wig_fluid_last_error(void);

/* Library ABI version (WIG_ABI_VERSION). */
uint32_t wig_fluid_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* WIG_FLUID_H */
