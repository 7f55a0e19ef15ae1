// wig_device.cuh — device-side layout, constants and helpers of the liquid
// step.  Every buffer is in the reference's layout (shaders/fluid.wgsl:85-181,
// js/sim.js:741-843); the helpers here are the addressing and cell-word
// accessors those layouts imply (fluid.wgsl:246-327, common.wgsl:5-270,
// js/shared.js:63-110).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/wig_fluid.h"

namespace wig {

// The message wig_fluid_last_error() returns on this thread.
void set_last_error(const std::string& msg);

// ---------------------------------------------------------------- constants
constexpr uint32_t NONE = 0xffffffffu;
constexpr uint32_t G_COUNT = 0, G_TAKEN = 1, G_SORT = 2, G_START = 3, G_DEST = 4, G_TYPE = 5,
                   G_DENSITY = 6, G_MASS = 7, G_AIR_TO = 8, G_RIM = 9;
constexpr uint32_t G_REGION = G_TAKEN, G_CAME = G_TAKEN;
constexpr uint32_t CELL_WORDS = 11;
constexpr float FIX = 65536.0f;
constexpr int BLOCK = 8;
constexpr uint32_t MARK_LIQUID = 1, MARK_REGION = 2;
constexpr uint32_t ACTIVE = 1, HAS_FLUID = 2, HAS_VISCOUS = 4, NEAR_LIQUID = 8;
constexpr float SMOOTH_OMEGA = 1.0f, OMEGA = 1.8f, VISC_OMEGA = 1.6f;
constexpr float SPREAD = 0.3f, MAX_DRIFT = 0.5f, DRIFT_KEEP = 0.9f, PROJECTED = 2.0f;
constexpr float AFFINE_KEEP = 0.95f, LIQUID_MAX_SPEED = 8.0f;
constexpr int ADVECT_STEPS = 17;
constexpr float IMPACT_SPEED = 2.5f;
constexpr float THETA_MIN = 0.1f;
constexpr float APART = 1.0f / 256.0f, APART_FIX = 16777216.0f;
constexpr float LIQUID_TOLERANCE = 1e-2f;
constexpr int RIM = BLOCK + 2, SWEEPS = 4, COARSE_SWEEPS = 40;
constexpr uint32_t REGION_OPEN = 0x80000000u;
constexpr float PIN = 1.0f;
constexpr uint32_t CAME_PRESSING = 1, CAME_FALLING = 2;
constexpr int COLUMN_MOST = 512, ESCAPE_REACH = 16;
constexpr uint32_t DEST_KEEP = 0xffffffffu, DEST_ASIDE = 0x80000000u, DEST_CELL = 0x40000000u,
                   DEST_SPAN = 0x3fffffffu;
constexpr uint32_t LIQUID_COUNT_BITS = 8, LIQUID_COUNT_MAX = 255;
constexpr uint32_t FL_BURN = 1, FL_DRAWN = 4, FLAG_SHIFT = 28;
constexpr uint32_t F_IMPACT = 32;
constexpr float POWDER_PUSH = 0.3f, BUBBLE_GAS = 0.25f, SLIP = 1.0f;
constexpr uint32_t RASTER_KINDS = 4;
constexpr float EXACT_FINE = 4294967296.0f;
constexpr float AMBIENT_T = 20.0f;
constexpr uint32_t AIR = WIG_ELEM_AIR, WATER = WIG_ELEM_WATER;
constexpr uint32_t COUNT_ACTIVE = 0, COUNT_RETIRED = 1, COUNT_VISCOUS = 2, COUNT_PARTICLES = 3,
                   COUNT_RESIDUAL = 4, COUNT_CYCLES = 7, COUNT_MOST_CYCLES = 8;
// A bound on any lock-free retry loop (the union-find's): past it the
// kernel records WIG_ERR_LOOP in the step's error word and gives up.
constexpr uint32_t LOOP_LIMIT = 1u << 22;
constexpr uint32_t ERR_LOOP = 1u, ERR_CAPACITY = 2u, ERR_BARRIER = 4u;
// A grid barrier's wait: at most this many polls of ~64 ns (about half a
// second), past which the kernel records ERR_BARRIER and returns.
constexpr uint32_t BARRIER_SPIN_LIMIT = 1u << 23;
// The bounds in force on a device (the two above unless
// wig_fluid_set_wait_limits lowered them, which the failure-path tests do to
// see the error come back); read by the loops at run time.
extern __device__ uint32_t g_loop_limit;
extern __device__ uint32_t g_spin_limit;

// What the host writes for a world before each step: its Params, the
// solve's stopping rule, and its part of the step (a batch steps worlds with
// different flags): bookkeeping only, viscosity sweeps, the tiling the
// step's first relaxation is on.
struct StepHead {
    wig_params P;
    uint32_t tol_mode;
    uint32_t f64;
    uint32_t book;
    uint32_t viscous;
    uint32_t shift_first;
    uint32_t pad_;
    double tol;
};

// Per-step state of a world in device memory: its head, then the solve's
// scalars (tolerance form and FP64 dots), set by the step itself.  Read by
// every kernel, so a captured graph replays with new values.
struct StepState {
    wig_params P;
    uint32_t tol_mode;
    uint32_t f64;
    uint32_t book;
    uint32_t viscous;
    uint32_t shift_first;
    uint32_t pad_;
    double tol;
    // set at the step's start: error word, residuals
    uint32_t err;
    uint32_t cycles_run;
    double rel;
    double bnorm2;
    double rz;
    double pq;
    double alpha;
    double beta;
    // the fast form's iteration count, loop decision, last-block counters and
    // f32 scalars (fluid.wgsl's cg sums: r.z, alpha, beta, p.Ap)
    uint32_t cycle;
    uint32_t cont;
    uint32_t fdone[6];
    uint32_t check;     // the mixed form: this iteration's true residual is to be checked
    uint32_t drift;     // the mixed form: the true residual is to be put in for the recursive one
    double rel_true;    // the mixed form: the last check's ||b + A x||2/||b||2
    float rz32, pq32, alpha32, beta32;
    // the persistent solve's grid barrier: arrivals and generation
    uint32_t bar_count;
    uint32_t bar_gen;
};
static_assert(sizeof(StepHead) == offsetof(StepState, err), "StepHead is StepState's prefix");

// A world and its buffers (an entry of a batch's world table).
struct Dev {
    int W, H;
    uint32_t C, F, B, BW, BH, cap, ppc, edge_tiles, levels;
    uint32_t bw_mul;  // floor((2^32 - 1) / BW): a block index's row by a multiply-high and one correction
    uint32_t level_w[WIG_MG_LEVELS + 1];
    uint32_t level_h[WIG_MG_LEVELS + 1];
    uint32_t level_start[WIG_MG_LEVELS + 1];
    uint32_t* cells;
    uint32_t* sorted;
    uint32_t* parts;
    uint32_t* counters;
    float* field;
    uint32_t* blocks;
    float* cg;
    const wig_elem* elems;
    uint32_t n_elems;
    StepState* st;
    double* part64;   // 2 doubles per block: FP64 partial sums
    double* norm64;   // 2 doubles per block: FP64 norms' partials
    uint32_t* motion; // binding 12, the free bodies' table (null: no free bodies)
    uint32_t* pushes; // binding 16, the solve's exact sums of what it does to each body
    uint32_t* stamps; // binding 14, the bodies' buffer, read for its swept stamps (null: no seams or cups)
};

struct I2 { int x, y; };
struct V2 { float x, y; };

// ---------------------------------------------------------------- WGSL semantics
__device__ __forceinline__ int32_t f2i(float f) { return __float2int_rz(f); }     // saturating, NaN -> 0
__device__ __forceinline__ uint32_t f2u(float f) { return __float2uint_rz(f); }  // saturating, < 0 -> 0
__device__ __forceinline__ float rnd_even(float x) { return rintf(x); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float len2(float x, float y) { return __fsqrt_rn(x * x + y * y); }

// a / d rounded to float (IEEE, round to nearest even) for a divisor d that
// divides many times: quotBy(a, recipOf(d)) is a times the FP64 reciprocal
// of d, rounded to float.  Why it is the quotient's bits:
// - recipOf(d) = (1/d)(1 + e1) and the FP64 product (a/d)(1 + e1)(1 + e2),
//   |e1|, |e2| <= 2^-53: within 2^-51.9 of a/d, relative.
// - With a = A 2^i and d = D 2^k (A, D < 2^24 integers), a float rounding
//   boundary m near a/d (a midpoint between two floats, the overflow
//   threshold, or a subnormal midpoint) has a - d m a multiple of
//   2^min(i, k + ulp exponent), so a/d is at least 2^-49 from m, relative,
//   or 2^-174 absolute below the normal range, and never on m (d m would
//   need an odd factor above 2^24 that A lacks).
// - So no boundary lies between a/d and the product: both round to the
//   same float.  Zeros, infinities and NaNs follow IEEE's products as the
//   quotient's special cases do (1/0 = inf, 0 inf = NaN, a / inf = a 0).
// The method is this bound on the gap between a quotient of p-bit numbers
// and the rounding points (the argument of double-rounding results for
// division with a 2p + 2-bit intermediate format), checked in the tests
// against the GPU's and the host's IEEE division on random bit patterns.
__device__ __forceinline__ double recipOf(float d) { return 1.0 / (double)d; }
__device__ __forceinline__ float quotBy(float a, double rd) { return __double2float_rn((double)a * rd); }

__device__ __forceinline__ float f16_value(uint32_t h) { return __half2float(__ushort_as_half((unsigned short)h)); }
__device__ __forceinline__ uint32_t pack2x16(float a, float b) {
    return (uint32_t)__half_as_ushort(__float2half_rn(a)) | ((uint32_t)__half_as_ushort(__float2half_rn(b)) << 16);
}

__device__ __forceinline__ uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
struct Rng {
    uint32_t s;
    __device__ void seed(uint32_t a, uint32_t b, uint32_t c) { s = pcg(a ^ pcg(b ^ pcg(c))); }
    __device__ float next() { s = pcg(s); return (float)(s >> 8u) * (1.0f / 16777216.0f); }
};

// sin and cos of a in [0, 2 pi): Cody-Waite reduction by pi/2 and Taylor
// series on [-pi/4, pi/4], the same arithmetic as the oracle's.
__device__ __forceinline__ void sincos_own(float a, float* s, float* c) {
    float k = rintf(a * 0.636619772f);
    float r = (a - k * 1.57079637f) - k * -4.37113883e-8f;
    float r2 = r * r;
    float sp = r * (1.0f + r2 * (-0.166666667f + r2 * (0.00833333333f + r2 * (-0.000198412698f + r2 * 2.75573192e-6f))));
    float cp = 1.0f + r2 * (-0.5f + r2 * (0.0416666667f + r2 * (-0.00138888889f + r2 * 2.48015873e-5f)));
    int q = ((int)k) & 3;
    if (q == 0) { *s = sp; *c = cp; }
    else if (q == 1) { *s = cp; *c = -sp; }
    else if (q == 2) { *s = -sp; *c = -cp; }
    else { *s = -cp; *c = sp; }
}

// Word fields (js/shared.js:79).
__device__ __forceinline__ uint32_t wordType(uint32_t x) { return x & 0xffu; }
__device__ __forceinline__ uint32_t wordAux(uint32_t x) { return (x >> 8) & 0xffu; }
__device__ __forceinline__ uint32_t wordLife(uint32_t x) { return (x >> 16) & 0xffu; }
__device__ __forceinline__ uint32_t wordShade(uint32_t x) { return (x >> 24) & 0xfu; }
__device__ __forceinline__ uint32_t wordFlags(uint32_t x) { return x >> 28; }
__device__ __forceinline__ uint32_t packWord(uint32_t t, uint32_t aux, uint32_t life, uint32_t shade, uint32_t flags) {
    return (t & 0xffu) | ((aux & 0xffu) << 8) | ((life & 0xffu) << 16) | ((shade & 0xfu) << 24) | ((flags & 0xfu) << 28);
}
__device__ __forceinline__ uint32_t wordWith(uint32_t x, uint32_t f) { return x | (f << FLAG_SHIFT); }
__device__ __forceinline__ uint32_t wordWithout(uint32_t x, uint32_t f) { return x & ~(f << FLAG_SHIFT); }
__device__ __forceinline__ bool wordHas(uint32_t x, uint32_t f) { return (wordFlags(x) & f) != 0u; }
__device__ __forceinline__ bool holdsSolute(uint32_t t) { return t == WATER; }
__device__ __forceinline__ uint32_t wordSolute(uint32_t x) { return holdsSolute(wordType(x)) ? wordAux(x) : 0u; }
__device__ __forceinline__ uint32_t wordStrength(uint32_t x) { return holdsSolute(wordType(x)) ? wordLife(x) : 0u; }
__device__ __forceinline__ uint32_t liquidHome(uint32_t w) { return w >> LIQUID_COUNT_BITS; }
__device__ __forceinline__ uint32_t liquidCount(uint32_t w) { return w & LIQUID_COUNT_MAX; }
__device__ __forceinline__ uint32_t liquidW(uint32_t home, uint32_t count) {
    return (home << LIQUID_COUNT_BITS) | min(count, LIQUID_COUNT_MAX);
}
__device__ __forceinline__ uint32_t claimOf(uint32_t i) { return DEST_CELL | (DEST_SPAN - i); }
__device__ __forceinline__ uint32_t claimedCell(uint32_t d) { return DEST_SPAN - (d & DEST_SPAN); }
__device__ __forceinline__ bool isClaim(uint32_t d) { return d != DEST_KEEP && (d & DEST_ASIDE) == 0u && (d & DEST_CELL) != 0u; }
__device__ __forceinline__ uint32_t drawnAs(uint32_t word) { return wordType(word) | (wordAux(word) << 8); }
__device__ __forceinline__ uint32_t takenBy(uint32_t i) { return ~i; }

__device__ __forceinline__ I2 beside(I2 c, int d) {
    return d < 2 ? I2{c.x + (d & 1) * 2 - 1, c.y} : I2{c.x, c.y + (d & 1) * 2 - 1};
}

// ---------------------------------------------------------------- the world, device side
struct W {
    const Dev& D;
    __device__ explicit W(const Dev& d) : D(d) {}

    __device__ bool inWorld(I2 c) const { return c.x >= 0 && c.y >= 0 && c.x < D.W && c.y < D.H; }
    __device__ uint32_t cellIndex(I2 c) const { return (uint32_t)c.y * (uint32_t)D.W + (uint32_t)c.x; }
    __device__ I2 cellOf(float px, float py) const {
        int x = f2i(floorf(px)), y = f2i(floorf(py));
        return I2{min(max(x, 0), D.W - 1), min(max(y, 0), D.H - 1)};
    }
    __device__ uint32_t uFace(int x, int y) const { return (uint32_t)y * (uint32_t)(D.W + 1) + (uint32_t)x; }
    __device__ uint32_t vFace(int x, int y) const {
        return (uint32_t)(D.W + 1) * (uint32_t)D.H + (uint32_t)y * (uint32_t)D.W + (uint32_t)x;
    }
    __device__ bool faceInWorld(I2 at, bool isU) const {
        int ex = D.W + (isU ? 1 : 0), ey = D.H + (isU ? 0 : 1);
        return at.x >= 0 && at.y >= 0 && at.x < ex && at.y < ey;
    }
    __device__ uint32_t faceIndex(I2 at, bool isU) const { return isU ? uFace(at.x, at.y) : vFace(at.x, at.y); }

    // counters
    __device__ uint32_t* gwp(uint32_t i, uint32_t g) const { return D.counters + (size_t)CELL_WORDS * i + g; }
    __device__ uint32_t gw(uint32_t i, uint32_t g) const { return D.counters[(size_t)CELL_WORDS * i + g]; }
    __device__ uint32_t sumSlot(uint32_t f) const { return CELL_WORDS * D.C + 2u * f; }
    __device__ float densityAt(I2 c) const {
        if (!inWorld(c)) return 0.0f;
        return (float)gw(cellIndex(c), G_DENSITY) / (FIX * (float)D.ppc);
    }

    // field
    __device__ float* fv(uint32_t v) const { return D.field + 4u * (size_t)v; }
    __device__ float4 f4(uint32_t v) const { return reinterpret_cast<const float4*>(D.field)[v]; }
    __device__ float4 gridAt(I2 c) const {
        if (!inWorld(c)) return make_float4(0.0f, 0.0f, -1.0f, 0.0f);
        return f4(2u * cellIndex(c));
    }
    __device__ float driftAt(I2 c) const { return inWorld(c) ? fv(2u * cellIndex(c) + 1u)[0] : 0.0f; }
    __device__ uint32_t faceSlot(uint32_t f) const { return 2u * D.C + f; }
    __device__ float* viscRhsP(uint32_t f) const { return fv(faceSlot(D.F + f / 4u)) + f % 4u; }
    __device__ float* viscLastP(uint32_t f) const { return fv(faceSlot(D.F + (D.F + 3u) / 4u + f / 4u)) + f % 4u; }

    // blocks
    __device__ bool inBlocks(I2 b) const { return b.x >= 0 && b.y >= 0 && b.x < (int)D.BW && b.y * (int)D.BW < (int)D.B; }
    __device__ uint32_t blockIndex(I2 b) const { return (uint32_t)b.y * D.BW + (uint32_t)b.x; }
    __device__ uint32_t stateSlot(uint32_t n) const { return D.B + n; }
    __device__ uint32_t activeSlot(uint32_t n) const { return 2u * D.B + n; }
    __device__ uint32_t retiredSlot(uint32_t n) const { return 3u * D.B + n; }
    __device__ uint32_t countSlot(uint32_t w) const { return 4u * D.B + w; }
    __device__ uint32_t totalSlot(uint32_t n) const { return 4u * D.B + WIG_FLUID_STATS + n; }
    __device__ uint32_t activeCount() const { return D.blocks[countSlot(COUNT_ACTIVE)]; }
    __device__ bool isActiveBlock(I2 b) const { return inBlocks(b) && (D.blocks[stateSlot(blockIndex(b))] & ACTIVE) != 0u; }
    __device__ uint32_t statesOf(I2 b0, I2 b1) const {
        uint32_t r = 0;
        for (int y = b0.y; y <= b1.y; y++)
            for (int x = b0.x; x <= b1.x; x++)
                if (inBlocks(I2{x, y})) r |= D.blocks[stateSlot(blockIndex(I2{x, y}))];
        return r;
    }
    // Block n's (column, row): n / BW as umulhi(n, floor((2^32 - 1) / BW)),
    // which is the quotient or one below it for any 32-bit n, corrected by
    // the remainder (in place of an integer division's instruction sequence).
    __device__ __forceinline__ I2 blockAt(uint32_t n) const {
        uint32_t q = __umulhi(n, D.bw_mul), r = n - q * D.BW;
        if (r >= D.BW) {
            q += 1u;
            r -= D.BW;
        }
        return I2{(int)r, (int)q};
    }
    __device__ I2 activeBlock(uint32_t wid) const { return blockAt(D.blocks[activeSlot(wid)]); }
    // facesOf (fluid.wgsl:296-303)
    __device__ void facesOf(I2 c, int out[4][3]) const {
        bool right = c.x == D.W - 1 || (c.x % BLOCK == BLOCK - 1 && !isActiveBlock(I2{c.x / BLOCK + 1, c.y / BLOCK}));
        bool bottom = c.y == D.H - 1 || (c.y % BLOCK == BLOCK - 1 && !isActiveBlock(I2{c.x / BLOCK, c.y / BLOCK + 1}));
        out[0][0] = c.x; out[0][1] = c.y; out[0][2] = 1;
        out[1][0] = c.x; out[1][1] = c.y; out[1][2] = 0;
        out[2][0] = c.x + 1; out[2][1] = c.y; out[2][2] = right ? 1 : -1;
        out[3][0] = c.x; out[3][1] = c.y + 1; out[3][2] = bottom ? 0 : -1;
    }

    // particles
    __device__ uint4* items(uint32_t* buf) const { return reinterpret_cast<uint4*>(buf + 4); }

    // cells
    __device__ uint4 cell(uint32_t i) const { return reinterpret_cast<const uint4*>(D.cells)[i]; }
    __device__ uint32_t cellType(uint32_t i) const { return wordType(D.cells[4u * (size_t)i]); }
    __device__ const wig_elem& elem(uint32_t t) const { return D.elems[t < D.n_elems ? t : 0u]; }
    __device__ uint32_t kindOf(uint32_t t) const { return elem(t).kind; }
    __device__ uint32_t kindOfCell(uint32_t i) const { return kindOf(cellType(i)); }
    __device__ uint32_t* gasPairPtr(uint32_t i) const {
        return D.cells + 4u * (size_t)(D.C + (i >> 1u)) + ((i & 1u) ? 2u : 0u);
    }
    __device__ float gasAmountOf(uint32_t i) const { return f16_value(gasPairPtr(i)[1] >> 16); }

    // gravity: the Earth's pull alone, down +y (pull.wgsl:31-46, no masses' field)
    __device__ V2 pull() const { return V2{0.0f + 0.0f, D.st->P.earth_g + 0.0f}; }

    // elements (common.wgsl:981-997, :1469-1564)
    __device__ float actsAt(uint32_t x, float temp) const {
        const wig_elem& e = elem(wordType(x));
        return clampf(temp, e.lo_t, e.hi_t) + fmaxf(temp - e.hi_t - e.up_span, 0.0f)
            - fmaxf(e.lo_t - e.down_span - temp, 0.0f) * e.down_scale;
    }
    __device__ float expandedAt(uint32_t t, float temp) const {
        const wig_elem& e = elem(t);
        float d = temp - fmaxf(AMBIENT_T, e.lo_t);
        return clampf(1.0f - e.expansion * d - e.expansion2 * d * d, 0.8f, 1.05f);
    }
    __device__ float liquidDensity(uint32_t x, float temp) const {
        uint32_t t = wordType(x);
        uint32_t solute = wordSolute(x);
        float acts = actsAt(x, temp);
        float density = elem(t).density / 100.0f * expandedAt(t, acts);
        if (holdsSolute(t) && solute != 0u) density += elem(solute).sol_density * ((float)wordStrength(x) / 255.0f);
        return density;
    }
    __device__ float liquidVolume(uint32_t x, float temp) const {
        return 1.0f / expandedAt(wordType(x), actsAt(x, temp));
    }
    __device__ float viscosityAt(const wig_elem& e, float temp) const {
        if (e.viscosity_e <= 0.0f) return e.viscosity;
        return fminf(e.viscosity * expf((e.viscosity_t - temp) / e.viscosity_e), 1e4f);
    }

    __device__ bool converged(uint32_t cycle) const {
        if (D.st->tol_mode) return cycle > 0u && D.st->rel <= D.st->tol;
        uint32_t slot = countSlot(COUNT_RESIDUAL + (cycle + 2u) % 3u);
        return cycle > 0u && __uint_as_float(D.blocks[slot]) < LIQUID_TOLERANCE;
    }
};

// faceBeta, surfaceShare, fineBeta (fluid.wgsl:369-405)
__device__ __forceinline__ float faceBeta(float a, float b) {
    if (a < 0.0f || b < 0.0f || (a <= 0.0f && b <= 0.0f)) return 0.0f;
    return (a > 0.0f && b > 0.0f) ? 2.0f / (a + b) : 1.0f / fmaxf(a, b);
}
__device__ __forceinline__ float surfaceShare(float da, float db) {
    return clampf((da - 0.5f) / fmaxf(da - db, 1e-3f), THETA_MIN, 1.0f);
}
__device__ __forceinline__ float fineBeta(float a, float b, float da, float db) {
    float beta = faceBeta(a, b);
    if (a > 0.0f && b == 0.0f) return beta / (da > 0.0f ? surfaceShare(da, db) : 0.5f);
    if (b > 0.0f && a == 0.0f) return beta / (db > 0.0f ? surfaceShare(db, da) : 0.5f);
    return beta;
}

// ---------------------------------------------------------------- batches

// One multigrid level's arrays in the fast form's scratch, a float per cell
// (row-major, the level's width): potentials and right-hand sides (pressure
// x, drift y), density, and the stencil's coefficients to the left, right,
// upper and lower neighbours (0 past an obstacle or the edge) with their sum.
struct Lvl {
    float *px, *py, *rx, *ry, *rho;
    float *b0, *b1, *b2, *b3, *diag;
    float *ux, *uy;  // levels >= 1: the potentials after the V-cycle's way up (the way down's stay in px, py)
};

// A level's operator in binary16 (the mixed-precision form), n values an
// array from base: on a coarse level its density and four stencil
// coefficients (rho, b0, b1, b2, b3), whose potentials and right-hand sides
// are stored as bf16 in the first half of Lvl's f32 arrays; on level 0 the
// four coefficients alone, the copies the smoother reads (the CG's A p reads
// Lvl's f32 ones).
struct LvlH {
    __half* base;
    uint32_t n;
    uint32_t pad_;
};

// A world's fast-form scratch.
struct FastW {
    Lvl L[WIG_MG_LEVELS + 1];  // level 0 (the cells) .. levels
    LvlH H[WIG_MG_LEVELS + 1]; // the operator in binary16 (the mixed form): level 0's coefficients, levels 1 ..
    float* pin;                // level 0: PIN at a pinned root, else 0
    uint8_t* fmask;            // level 0: bit d set when neighbour d is liquid
    float *rimx, *rimy;        // level 0: the relaxation's rim snapshot
    float *X, *R, *P, *Q;      // level 0: CG's x, r, p, A p
    float* P2;                 // level 0: p of the fast form's odd iterations (p of the even ones in P)
    float* part32;             // 2 per block
    double* part64;            // 2 per block
    uint32_t lc;               // first level the one-CTA coarse kernel solves
    uint32_t lp;               // first level CTA 0 of the persistent solve holds
};

// An entry of a batch's world table (device memory).
struct alignas(16) World {
    Dev D;
    FastW S;
};
static_assert(sizeof(World) % 16 == 0, "World copies in 16-byte words");

// Work lists.  A kernel's CTAs take the items of one list in turn (grid
// stride); an item is a world of the batch (its index in the world table, the
// high bits) and a unit of that world's work (the low Batch::lbits bits):
// The 16x16 tiles of a w x h level: the units of the level lists.
__host__ __device__ __forceinline__ uint32_t levelTiles(uint32_t w, uint32_t h) {
    return ((w + 15u) / 16u) * ((h + 15u) / 16u);
}

enum List : uint32_t {
    L_WB = 0,     // every 8x8 block of the world (sync, syncSeed)
    L_PS,         // 256 particles of `sorted` (syncParticles)
    L_PP,         // 256 particles of `parts` (gather, advect, sortCount, scatter)
    L_ACT,        // an active block (the passes over the blocks worked on)
    L_RET,        // a retired block
    L_ACT4,       // four active blocks (the fast form's 256-thread CG kernels)
    L_RELAX,      // a relaxation tile: the active blocks, then the shifted tiling's edge tiles
    L_ONE_ALL,    // the world (per-world single-CTA work: compact, report)
    L_ONE,        // the world when it runs the full step (scanTotals, the coarse levels, ...)
    L_RES,        // + l - 1: 16x16 tiles of level l when the fast form restricts it by itself (l <= lc)
    L_SM = L_RES + WIG_MG_LEVELS,  // + l - 1: 16x16 tiles of level l below the coarse kernel's (l < lc)
    L_COUNT = L_SM + WIG_MG_LEVELS
};

// A batch as every kernel sees it: the world table and the work lists
// (list L's items at items + base[L], count[L] of them, written on the
// device by the schedule kernels).
struct Batch {
    const World* __restrict__ worlds;
    const uint32_t* __restrict__ items;
    const uint32_t* __restrict__ count;
    uint32_t base[L_COUNT];
    uint32_t lbits;           // bits of an item's unit
    uint32_t single;          // a batch of one world: item g of any list is unit g of world 0
    uint32_t mixed;           // the mixed-precision form (coarse operators in binary16, true-residual checks)
    uint32_t max_cycles;
    unsigned long long cond;  // cudaGraphConditionalHandle of the iteration loop (0: none)
    unsigned long long cond_check;  // the mixed form's IF node of the true-residual check (0: none)
    unsigned long long cond_drift;  // the IF node of its fix (0: none)
    uint32_t* loop;           // the loop's verdict: 1 when a world iterates again

    __device__ __forceinline__ uint32_t n(uint32_t list) const { return count[list]; }
    __device__ __forceinline__ uint32_t item(uint32_t list, uint32_t g) const {
        return single ? g : items[base[list] + g];
    }
    __device__ __forceinline__ const World& world(uint32_t it) const { return worlds[(uint64_t)it >> lbits]; }
    __device__ __forceinline__ uint32_t unit(uint32_t it) const { return it & ((1u << lbits) - 1u); }
};

// The CTAs of a kernel over list L, one item per CTA at a time, each CTA a
// contiguous run of the list (so its items are mostly of one world):
//   FOR_ITEMS(Bt, L, it) { const World& Wd = Bt.world(it); uint32_t j = Bt.unit(it); ... }
#define FOR_ITEMS(Bt, L, it)                                                                       \
    for (uint32_t n_##it = (Bt).n(L), p_##it = (n_##it + gridDim.x - 1u) / gridDim.x,              \
                  g_##it = blockIdx.x * p_##it, e_##it = min(g_##it + p_##it, n_##it), it = 0;     \
         g_##it < e_##it && ((it = (Bt).item((L), g_##it)), true); g_##it++)
// A CTA's copy of the world of its current item, in shared memory: copied
// when the item's world changes (uniformly across the CTA), so the world's
// fields cost a shared-memory read instead of a chain of global loads.
struct WorldCopy {
    World w;
    uint32_t k;
};
__device__ __forceinline__ void worldCopyInit(WorldCopy& c) {
    if (threadIdx.x == 0) c.k = 0xffffffffu;
    __syncthreads();
}
__device__ __forceinline__ const World& worldOf(const Batch& Bt, uint32_t it, WorldCopy& c) {
    const uint32_t k = (uint32_t)((uint64_t)it >> Bt.lbits);
    if (k != c.k) {
        __syncthreads();  // the CTA is done with the last world's copy
        const uint4* src = reinterpret_cast<const uint4*>(&Bt.worlds[k]);
        uint4* dst = reinterpret_cast<uint4*>(&c.w);
        for (uint32_t i = threadIdx.x; i < sizeof(World) / 16u; i += blockDim.x) dst[i] = src[i];
        if (threadIdx.x == 0) c.k = k;  // read again only after the barrier below
        __syncthreads();
    }
    return c.w;
}

// An item's world D (with its accessors w) and unit j, read from the world
// table (any thread, any loop).
#define ITEM_WORLD(Bt, it, D, w, j)              \
    const Dev& D = (Bt).world(it).D;             \
    const W w(D);                                \
    const uint32_t j = (Bt).unit(it)
// The same from the CTA's copy (every thread of the CTA, each item in turn;
// the kernel declares `__shared__ WorldCopy wc_;` and calls worldCopyInit).
#define ITEM_WORLD_C(Bt, it, D, w, j)            \
    const Dev& D = worldOf((Bt), (it), wc_).D;   \
    const W w(D);                                \
    const uint32_t j = (Bt).unit(it)

}  // namespace wig
