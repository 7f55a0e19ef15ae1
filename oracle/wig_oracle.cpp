// wig_oracle.cpp — TEST INFRASTRUCTURE: the CPU oracle of the liquid step.
//
// This file is the checker, not the product.  Only tests/, the smoke check
// and bench.py's CPU-baseline leg may load it.  It restates, pass by pass,
// the reference's liquid step (shaders/fluid.wgsl, dispatched in the order of
// Simulation.encodeFluid, js/sim.js:2466-2612) over the reference's own
// buffer layouts, single-threaded and in plain IEEE f32 arithmetic (built
// with -ffp-contract=off, so no multiply-add is fused).  Each function cites
// the WGSL it follows.
//
// Parity pin: the reference ships no test vectors for this path (its
// test/*.mjs scripts are named in comments but absent), and its arithmetic
// runs in a browser's WebGPU, which is not present here.  The oracle is
// pinned instead by the invariants the reference's scenes state (a dam break
// loses no particle, js/scenes.js:1089; a still tank comes to rest with its
// pressure growing with depth, js/scenes.js:1085, fluid.wgsl:1566-1575), by
// the integer invariants of the splat, and by an FP64 solve of the same
// operator.
//
// Scope: the element subset AIR, WALL, WATER (and any element table given),
// no air motion (binding 3 unbound: no air push in gather, no wind drag in
// setFace), free bodies only when their table and sums are bound (bindings
// 12 and 16, wo_bind_bodies; else rigidAt and heldAt are NONE) and their
// seams and cups only when the bodies' buffer is too (binding 14; else
// seamOf, cupOf and cupBefore are NONE), no people (binding 13 unbound: isOccupant is false), and
// the Earth's pull alone (binding 10 unbound: pullAt = (0, P.earthG), down is
// +y).  Surface tension's pass runs only when sim.js's surfaceTension() holds
// (capillary length over dx >= 0.3 cells), which no config reaches.

#include "../include/wig_fluid.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

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
constexpr float AMBIENT_T = 20.0f, KELVIN = 273.15f;
constexpr uint32_t AIR = WIG_ELEM_AIR, WATER = WIG_ELEM_WATER;
constexpr uint32_t COUNT_ACTIVE = 0, COUNT_RETIRED = 1, COUNT_VISCOUS = 2, COUNT_PARTICLES = 3,
                   COUNT_RESIDUAL = 4, COUNT_CYCLES = 7, COUNT_MOST_CYCLES = 8;
constexpr float VAPOUR_SCALE = 0.0f;  // vapour in the gas plane is not modelled (none in the configs)

// ---------------------------------------------------------------- WGSL semantics

inline uint32_t bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float flt(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline float rnd_even(float x) { return std::nearbyint(x); }  // WGSL round: half to even
// WGSL f32 -> i32: truncate toward zero, saturating; NaN gives 0.
inline int32_t f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483648.0f) return 2147483647;
    if (f <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)f;
}
inline uint32_t f2u(float f) {
    if (f != f || f <= 0.0f) return 0u;
    if (f >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)f;
}
// WGSL's min and max: of two f32, a NaN operand gives the other one (as the
// GPU's fminf and fmaxf do), otherwise the smaller or larger; any other type
// as std::min and std::max.
template <class T> inline T wmax(T a, T b) { return std::max(a, b); }
template <class T> inline T wmin(T a, T b) { return std::min(a, b); }
inline float wmax(float a, float b) { return a != a ? b : (b != b ? a : std::max(a, b)); }
inline float wmin(float a, float b) { return a != a ? b : (b != b ? a : std::min(a, b)); }
inline float clampf(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

// IEEE binary16 from f32, rounding to nearest even (pack2x16float).
uint16_t f16_bits(float f) {
    uint32_t x = bits(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // rounds past 65504
    if (ax < 0x38800000u) {  // below 2^-14: subnormal or zero
        if (ax < 0x33000000u) return (uint16_t)sign;  // under half the smallest subnormal
        uint32_t e = ax >> 23;
        uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        uint32_t shift = 126u - e;  // m * 2^(e-150) in units of 2^-24
        uint32_t q = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1u);
        if (rem > half || (rem == half && (q & 1u))) q++;
        return (uint16_t)(sign | q);
    }
    uint32_t e = (ax >> 23) - 127u + 15u;
    uint32_t m = ax & 0x7fffffu;
    uint32_t q = (e << 10) | (m >> 13);
    uint32_t rem = m & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q++;
    return (uint16_t)(sign | q);
}
float f16_value(uint32_t h) {
    uint32_t sign = (h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 31u, m = h & 1023u;
    if (e == 31u) return flt(sign | 0x7f800000u | (m << 13));
    if (e == 0u) {
        float v = (float)m * (1.0f / 16777216.0f);
        return sign ? -v : v;
    }
    return flt(sign | ((e - 15u + 127u) << 23) | (m << 13));
}
inline uint32_t pack2x16(float a, float b) { return (uint32_t)f16_bits(a) | ((uint32_t)f16_bits(b) << 16); }

// The pcg hash and generator (shaders/common.wgsl:1415-1432).
inline uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}

// sin and cos of a in [0, 2 pi) for pairWay: Cody-Waite reduction by pi/2 and
// Taylor series on [-pi/4, pi/4] (error under 2e-9 before rounding).
void sincos_own(float a, float* s, float* c) {
    float k = std::nearbyint(a * 0.636619772f);
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

struct I2 { int x, y; };
struct V2 { float x, y; };
struct V4 { float x, y, z, w; };
struct V3 { float x, y, z; };

// Word fields (js/shared.js:79): type [0,8), aux [8,16), life [16,24),
// shade [24,28), flags [28,32).
inline uint32_t wordType(uint32_t x) { return x & 0xffu; }
inline uint32_t wordAux(uint32_t x) { return (x >> 8) & 0xffu; }
inline uint32_t wordLife(uint32_t x) { return (x >> 16) & 0xffu; }
inline uint32_t wordShade(uint32_t x) { return (x >> 24) & 0xfu; }
inline uint32_t wordFlags(uint32_t x) { return x >> 28; }
inline uint32_t packWord(uint32_t t, uint32_t aux, uint32_t life, uint32_t shade, uint32_t flags) {
    return (t & 0xffu) | ((aux & 0xffu) << 8) | ((life & 0xffu) << 16) | ((shade & 0xfu) << 24) | ((flags & 0xfu) << 28);
}
inline uint32_t wordWith(uint32_t x, uint32_t f) { return x | (f << FLAG_SHIFT); }
inline uint32_t wordWithout(uint32_t x, uint32_t f) { return x & ~(f << FLAG_SHIFT); }
inline bool wordHas(uint32_t x, uint32_t f) { return (wordFlags(x) & f) != 0u; }
inline bool holdsSolute(uint32_t t) { return t == WATER; }
inline uint32_t wordSolute(uint32_t x) { return holdsSolute(wordType(x)) ? wordAux(x) : 0u; }
inline uint32_t wordStrength(uint32_t x) { return holdsSolute(wordType(x)) ? wordLife(x) : 0u; }
inline uint32_t liquidHome(uint32_t w) { return w >> LIQUID_COUNT_BITS; }
inline uint32_t liquidCount(uint32_t w) { return w & LIQUID_COUNT_MAX; }
inline uint32_t liquidW(uint32_t home, uint32_t count) { return (home << LIQUID_COUNT_BITS) | wmin(count, LIQUID_COUNT_MAX); }
inline uint32_t claimOf(uint32_t i) { return DEST_CELL | (DEST_SPAN - i); }
inline uint32_t claimedCell(uint32_t d) { return DEST_SPAN - (d & DEST_SPAN); }
inline bool isClaim(uint32_t d) { return d != DEST_KEEP && (d & DEST_ASIDE) == 0u && (d & DEST_CELL) != 0u; }
inline uint32_t drawnAs(uint32_t word) { return wordType(word) | (wordAux(word) << 8); }
inline uint32_t takenBy(uint32_t i) { return ~i; }

struct Particle {
    V2 pos, vel;
    uint32_t word;
    float temp;
    uint32_t id;
    V4 affine;
};

// ---------------------------------------------------------------- the world

struct Ctx {
    wig_world_layout L;
    const wig_params* P;
    const wig_elem* E;
    uint32_t nE;
    uint32_t* cells;
    uint32_t* sorted;
    uint32_t* parts;
    uint32_t* counters;
    float* field;
    uint32_t* blocks;
    float* cg;
    uint32_t* motion = nullptr;   // binding 12, the body table (null: no free bodies)
    uint32_t* pushes = nullptr;   // binding 16, the solve's sums of what it does to each body
    uint32_t* stamps = nullptr;   // binding 14, the bodies' buffer (its swept stamps; null: none)
    uint32_t level = 0, cycle = 0;
    uint32_t rng = 0;
    int W, H;
    uint32_t C, F, B, BW, cap, ppc;
    uint32_t levelStartV[WIG_MG_LEVELS + 1];
    // Tolerance form (WIG_STEP_TOLERANCE): the relative residual of the last
    // update and the tolerance; the residual slot test is replaced by it.
    bool tol_mode = false;
    bool f64_dots = false;
    double tol = 1e-6;
    double rel = 1.0;
    double bnorm2 = 0.0;

    const wig_elem& elem(uint32_t t) const { return E[t < nE ? t : 0]; }

    // addressing (fluid.wgsl:246-303)
    bool inWorld(I2 c) const { return c.x >= 0 && c.y >= 0 && c.x < W && c.y < H; }
    uint32_t cellIndex(I2 c) const { return (uint32_t)c.y * (uint32_t)W + (uint32_t)c.x; }
    I2 cellOf(V2 p) const {
        int x = f2i(std::floor(p.x)), y = f2i(std::floor(p.y));
        return I2{wmin(wmax(x, 0), W - 1), wmin(wmax(y, 0), H - 1)};
    }
    static I2 beside(I2 c, int d) {
        if (d < 2) return I2{c.x + (d & 1) * 2 - 1, c.y};
        return I2{c.x, c.y + (d & 1) * 2 - 1};
    }
    uint32_t uFace(int x, int y) const { return (uint32_t)y * (uint32_t)(W + 1) + (uint32_t)x; }
    uint32_t vFace(int x, int y) const { return (uint32_t)(W + 1) * (uint32_t)H + (uint32_t)y * (uint32_t)W + (uint32_t)x; }
    bool faceInWorld(I2 at, bool isU) const {
        int ex = W + (isU ? 1 : 0), ey = H + (isU ? 0 : 1);
        return at.x >= 0 && at.y >= 0 && at.x < ex && at.y < ey;
    }
    uint32_t faceIndex(I2 at, bool isU) const { return isU ? uFace(at.x, at.y) : vFace(at.x, at.y); }

    // counters (fluid.wgsl:307-327)
    uint32_t gridSlot(uint32_t i) const { return CELL_WORDS * i; }
    uint32_t sumSlot(uint32_t f) const { return CELL_WORDS * C + 2u * f; }
    uint32_t& gw(uint32_t i, uint32_t g) { return counters[gridSlot(i) + g]; }
    float densityAt(I2 c) {
        if (!inWorld(c)) return 0.0f;
        return (float)gw(cellIndex(c), G_DENSITY) / (FIX * (float)ppc);
    }
    float shareAt(I2 c) { return densityAt(c); }

    // field (fluid.wgsl:332-364)
    float* fv(uint32_t v) { return field + 4u * (size_t)v; }
    V4 gridAt(I2 c) {
        if (!inWorld(c)) return V4{0, 0, -1.0f, 0};
        float* f = fv(2u * cellIndex(c));
        return V4{f[0], f[1], f[2], f[3]};
    }
    float driftAt(I2 c) { return inWorld(c) ? fv(2u * cellIndex(c) + 1u)[0] : 0.0f; }
    uint32_t faceSlot(uint32_t f) const { return 2u * C + f; }
    float& viscRhs(uint32_t f) { return fv(faceSlot(F + f / 4u))[f % 4u]; }
    float& viscLast(uint32_t f) { return fv(faceSlot(F + (F + 3u) / 4u + f / 4u))[f % 4u]; }

    // blocks (fluid.wgsl:444-513)
    bool inBlocks(I2 b) const { return b.x >= 0 && b.y >= 0 && b.x < (int)BW && b.y * (int)BW < (int)B; }
    uint32_t blockIndex(I2 b) const { return (uint32_t)b.y * BW + (uint32_t)b.x; }
    uint32_t stateSlot(uint32_t n) const { return B + n; }
    uint32_t activeSlot(uint32_t n) const { return 2u * B + n; }
    uint32_t retiredSlot(uint32_t n) const { return 3u * B + n; }
    uint32_t countSlot(uint32_t w) const { return 4u * B + w; }
    uint32_t totalSlot(uint32_t n) const { return 4u * B + WIG_FLUID_STATS + n; }
    uint32_t activeCount() const { return blocks[countSlot(COUNT_ACTIVE)]; }
    bool isActiveBlock(I2 b) const { return inBlocks(b) && (blocks[stateSlot(blockIndex(b))] & ACTIVE) != 0u; }
    uint32_t statesOf(I2 b0, I2 b1) const {
        uint32_t r = 0;
        for (int y = b0.y; y <= b1.y; y++)
            for (int x = b0.x; x <= b1.x; x++)
                if (inBlocks(I2{x, y})) r |= blocks[stateSlot(blockIndex(I2{x, y}))];
        return r;
    }
    I2 activeBlock(uint32_t wid) const {
        uint32_t n = blocks[activeSlot(wid)];
        return I2{(int)(n % BW), (int)(n / BW)};
    }
    static I2 divI(I2 c, int k) { return I2{c.x / k, c.y / k}; }  // WGSL i32 division truncates

    // facesOf (fluid.wgsl:296-303): (x, y, isU) with isU < 0 for none.
    void facesOf(I2 c, int out[4][3]) const {
        bool right = c.x == W - 1 || (c.x % BLOCK == BLOCK - 1 && !isActiveBlock(I2{c.x / BLOCK + 1, c.y / BLOCK}));
        bool bottom = c.y == H - 1 || (c.y % BLOCK == BLOCK - 1 && !isActiveBlock(I2{c.x / BLOCK, c.y / BLOCK + 1}));
        out[0][0] = c.x; out[0][1] = c.y; out[0][2] = 1;
        out[1][0] = c.x; out[1][1] = c.y; out[1][2] = 0;
        out[2][0] = c.x + 1; out[2][1] = c.y; out[2][2] = right ? 1 : -1;
        out[3][0] = c.x; out[3][1] = c.y + 1; out[3][2] = bottom ? 0 : -1;
    }

    // particles (fluid.wgsl:517-538)
    uint32_t* item(uint32_t* buf, uint32_t k) { return buf + 4u + 4u * (size_t)k; }
    Particle toParticle(uint32_t* buf, uint32_t k) {
        uint32_t* m = item(buf, k);
        uint32_t* s = item(buf, cap + k);
        uint32_t* a = item(buf, 2u * cap + k);
        Particle q;
        q.pos = V2{flt(m[0]), flt(m[1])};
        q.vel = V2{flt(m[2]), flt(m[3])};
        q.word = s[0]; q.temp = flt(s[1]); q.id = s[2];
        q.affine = V4{flt(a[0]), flt(a[1]), flt(a[2]), flt(a[3])};
        return q;
    }
    void storeParticle(uint32_t k, const Particle& q) {
        uint32_t* m = item(parts, k);
        m[0] = bits(q.pos.x); m[1] = bits(q.pos.y); m[2] = bits(q.vel.x); m[3] = bits(q.vel.y);
        uint32_t* s = item(parts, cap + k);
        s[0] = q.word; s[1] = bits(q.temp); s[2] = q.id; s[3] = 0u;
        uint32_t* a = item(parts, 2u * cap + k);
        a[0] = bits(q.affine.x); a[1] = bits(q.affine.y); a[2] = bits(q.affine.z); a[3] = bits(q.affine.w);
    }
    uint32_t partsLive() const { return wmin(parts[0], cap); }

    // RNG (common.wgsl:1415-1432)
    void seedRng(uint32_t a, uint32_t b, uint32_t c) { rng = pcg(a ^ pcg(b ^ pcg(c))); }
    float rnd() { rng = pcg(rng); return (float)(rng >> 8u) * (1.0f / 16777216.0f); }

    // cells (common.wgsl cell accessors; js/shared.js:484-530)
    uint32_t* cellv(uint32_t i) { return cells + 4u * (size_t)i; }
    uint32_t cellType(uint32_t i) { return wordType(cells[4u * (size_t)i]); }
    uint32_t kindOfCell(uint32_t i) { return elem(cellType(i)).kind; }
    static float cellTemp(const uint32_t* v) { return flt(v[1]); }
    static V2 cellVel(const uint32_t* v) { return V2{f16_value(v[2] & 0xffffu), f16_value(v[2] >> 16)}; }
    // The gas plane (common.wgsl:412-460): cell i's pair at count + i/2.
    uint32_t* gasPairPtr(uint32_t i) { return cells + 4u * (size_t)(C + (i >> 1u)) + ((i & 1u) ? 2u : 0u); }
    float gasAmountOf(uint32_t i) {
        uint32_t* w = gasPairPtr(i);
        float vapour = f16_value(w[0] & 0xffffu);
        float amount = f16_value(w[1] >> 16);
        return amount + vapour * VAPOUR_SCALE;
    }

    // gravity (pull.wgsl:31-46) with no masses' field: the Earth's pull, down +y.
    V2 pullAt(V2) const { return V2{0.0f + 0.0f, P->earth_g + 0.0f}; }
    static I2 downAt(I2) { return I2{0, 1}; }

    // elements (common.wgsl:981-997, :1469-1564)
    float effTempIn(uint32_t t, float stored, float hiT, float loT) {
        const wig_elem& e = elem(t);
        return clampf(stored, loT, hiT) + wmax(stored - hiT - e.up_span, 0.0f)
            - wmax(loT - e.down_span - stored, 0.0f) * e.down_scale;
    }
    float actsAt(uint32_t x, float temp) {  // effTempIn(t, temp, phaseOf(t, solute, strength, 0))
        uint32_t t = wordType(x);
        const wig_elem& e = elem(t);
        return effTempIn(t, temp, e.hi_t, e.lo_t);
    }
    float expandedAt(uint32_t t, float temp) {
        const wig_elem& e = elem(t);
        float d = temp - wmax(AMBIENT_T, e.lo_t);
        return clampf(1.0f - e.expansion * d - e.expansion2 * d * d, 0.8f, 1.05f);
    }
    float liquidDensity(uint32_t x, float temp) {
        uint32_t t = wordType(x);
        uint32_t solute = wordSolute(x);
        float acts = actsAt(x, temp);
        float density = elem(t).density / 100.0f * expandedAt(t, acts);
        if (holdsSolute(t) && solute != 0u) {
            density += elem(solute).sol_density * ((float)wordStrength(x) / 255.0f);
        }
        return density;
    }
    float liquidVolume(uint32_t x, float temp) {
        uint32_t t = wordType(x);
        return 1.0f / expandedAt(t, actsAt(x, temp));
    }
    float viscosityAt(const wig_elem& e, float temp) {
        if (e.viscosity_e <= 0.0f) return e.viscosity;
        return wmin(e.viscosity * std::exp((e.viscosity_t - temp) / e.viscosity_e), 1e4f);
    }
    float wordTempOf(const uint32_t* v) { return actsAt(v[0], cellTemp(v)); }

    bool converged() {
        if (tol_mode) return cycle > 0u && rel <= tol;
        uint32_t slot = countSlot(COUNT_RESIDUAL + (cycle + 2u) % 3u);
        return cycle > 0u && flt(blocks[slot]) < LIQUID_TOLERANCE;
    }
};

// ---------------------------------------------------------------- the shared operator pieces

// faceBeta, surfaceShare, fineBeta (fluid.wgsl:369-405)
float faceBeta(float a, float b) {
    if (a < 0.0f || b < 0.0f || (a <= 0.0f && b <= 0.0f)) return 0.0f;
    return (a > 0.0f && b > 0.0f) ? 2.0f / (a + b) : 1.0f / wmax(a, b);
}
float surfaceShare(float da, float db) { return clampf((da - 0.5f) / wmax(da - db, 1e-3f), THETA_MIN, 1.0f); }
float fineBeta(float a, float b, float da, float db) {
    float beta = faceBeta(a, b);
    if (a > 0.0f && b == 0.0f) return beta / (da > 0.0f ? surfaceShare(da, db) : 0.5f);
    if (b > 0.0f && a == 0.0f) return beta / (db > 0.0f ? surfaceShare(db, da) : 0.5f);
    return beta;
}

// union-find over G_REGION words (label.wgsl:27-55)
uint32_t ufLink(Ctx& X, uint32_t at) { return X.gw(at, G_REGION); }
uint32_t ufFind(Ctx& X, uint32_t i) {
    uint32_t x = i;
    for (;;) {
        uint32_t up = ufLink(X, x);
        if (up >= x) break;
        x = up;
    }
    return x;
}
void ufJoin(Ctx& X, uint32_t i, uint32_t j) {
    uint32_t a = i, b = j;
    for (;;) {
        a = ufFind(X, a);
        b = ufFind(X, b);
        if (a == b) return;
        uint32_t lo = wmin(a, b), hi = wmax(a, b);
        uint32_t& w = X.gw(hi, G_REGION);
        uint32_t old = w;
        w = wmin(w, lo);
        if (old == hi) return;
        a = old;
        b = lo;
    }
}
bool pinnedAt(Ctx& X, uint32_t i) { return ufLink(X, i) == i; }

// Whether the cell at c (holding v) is in the liquid's way (fluid.wgsl:1120-1147).
bool fallingAt(Ctx& X, I2 q) {
    if (!X.inWorld(q)) return false;
    uint32_t fb = 4u << ((X.P->frame + 1u) & 1u);
    return (f2u(X.fv(2u * X.cellIndex(q) + 1u)[3]) & fb) != 0u;
}
bool isLiquidAt(Ctx& X, I2 c) { return X.inWorld(c) && X.kindOfCell(X.cellIndex(c)) == WIG_KIND_LIQUID; }
bool isObstacleCell(Ctx& X, I2 c) {
    uint32_t i = X.cellIndex(c);
    uint32_t t = X.cellType(i);
    uint32_t k = X.elem(t).kind;
    if (k == WIG_KIND_GAS) {
        int wet = 0;
        for (int d = 0; d < 4; d++) wet += isLiquidAt(X, Ctx::beside(c, d)) ? 1 : 0;
        if (wet < 2) return false;
        if (t == AIR) {
            I2 dn = Ctx::downAt(c);
            I2 up1{c.x - dn.x, c.y - dn.y}, up2{c.x - 2 * dn.x, c.y - 2 * dn.y};
            if (!isLiquidAt(X, up1) || !isLiquidAt(X, up2) || fallingAt(X, up1)) return false;
            return X.gasAmountOf(i) >= BUBBLE_GAS;
        }
        return true;
    }
    return k == WIG_KIND_SOLID || k == WIG_KIND_POWDER;
}
int countAt(Ctx& X, I2 c) {
    if (!X.inWorld(c)) return -1;
    uint32_t i = X.cellIndex(c);
    if (isObstacleCell(X, c)) return -1;
    return (int32_t)X.gw(i, G_COUNT);
}
// liquidIn (fluid.wgsl:1165-1179): (density, viscosity).
V2 liquidIn(Ctx& X, uint32_t i) {
    uint32_t* v = X.cellv(i);
    uint32_t t = wordType(v[0]);
    const wig_elem& e = X.elem(t);
    float acts = X.actsAt(v[0], Ctx::cellTemp(v));
    float viscosity = e.kind == WIG_KIND_LIQUID ? X.viscosityAt(e, acts) : 0.0f;
    uint32_t n = X.gw(i, G_COUNT);
    if (n > 0u) return V2{(float)X.gw(i, G_MASS) / (FIX * (float)n), viscosity};
    if (e.kind != WIG_KIND_LIQUID) return V2{1.0f, 0.0f};
    return V2{X.liquidDensity(v[0], Ctx::cellTemp(v)), viscosity};
}

// ---------------------------------------------------------------- levels

I2 levelSize(Ctx& X, uint32_t l) {
    return I2{(int)((((uint32_t)X.W) + ((1u << l) - 1u)) >> l), (int)((((uint32_t)X.H) + ((1u << l) - 1u)) >> l)};
}
bool inLevel(Ctx& X, uint32_t l, I2 c) {
    I2 s = levelSize(X, l);
    return c.x >= 0 && c.y >= 0 && c.x < s.x && c.y < s.y;
}
uint32_t levelSlot(Ctx& X, uint32_t l, I2 c) {
    I2 s = levelSize(X, l);
    return X.levelStartV[l] + 2u * ((uint32_t)c.y * (uint32_t)s.x + (uint32_t)c.x);
}
float rhoAt(Ctx& X, uint32_t l, I2 c) {
    if (!inLevel(X, l, c)) return -1.0f;
    if (l == 0u) return X.fv(2u * X.cellIndex(c))[2];
    return X.fv(levelSlot(X, l, c) + 1u)[0];
}
V2 potAt(Ctx& X, uint32_t l, I2 c) {
    if (!inLevel(X, l, c)) return V2{0, 0};
    if (l == 0u) {
        uint32_t i = 2u * X.cellIndex(c);
        return V2{X.fv(i)[0], X.fv(i + 1u)[0]};
    }
    float* f = X.fv(levelSlot(X, l, c));
    return V2{f[0], f[1]};
}
V2 rhsAt(Ctx& X, uint32_t l, I2 c) {
    if (l == 0u) {
        uint32_t i = 2u * X.cellIndex(c);
        return V2{X.fv(i)[1], X.fv(i + 1u)[1]};
    }
    float* f = X.fv(levelSlot(X, l, c));
    return V2{f[2], f[3]};
}
// stencil (fluid.wgsl:2286-2302)
void stencil(Ctx& X, uint32_t l, I2 c, float rho, V2* sum, float* diag) {
    V2 s{0, 0};
    float dg = 0.0f;
    for (int d = 0; d < 4; d++) {
        I2 n = Ctx::beside(c, d);
        float r = rhoAt(X, l, n);
        if (r < 0.0f) continue;
        float beta = faceBeta(rho, r);
        if (l == 0u) beta = fineBeta(rho, r, X.shareAt(c), X.shareAt(n));
        V2 p = potAt(X, l, n);
        s.x = s.x + beta * p.x;
        s.y = s.y + beta * p.y;
        dg = dg + beta;
    }
    *sum = s;
    *diag = dg;
}
// residualAt (fluid.wgsl:2306-2315)
V2 residualAt(Ctx& X, uint32_t l, I2 c) {
    float rho = rhoAt(X, l, c);
    if (rho <= 0.0f) return V2{0, 0};
    V2 sum; float diag;
    stencil(X, l, c, rho, &sum, &diag);
    float h2 = (float)(1u << (2u * l));
    float pinx = (l == 0u && pinnedAt(X, X.cellIndex(c))) ? PIN : 0.0f;
    V2 p = potAt(X, l, c), rhs = rhsAt(X, l, c);
    return V2{rhs.x - (sum.x - (diag + pinx) * p.x) / h2, rhs.y - (sum.y - (diag + 0.0f) * p.y) / h2};
}
// prolonged (fluid.wgsl:2478-2497)
V2 prolonged(Ctx& X, uint32_t l, I2 c) {
    I2 coarse{c.x / 2, c.y / 2};
    I2 s{(c.x & 1) == 1 ? 1 : -1, (c.y & 1) == 1 ? 1 : -1};
    const I2 off[4] = {{0, 0}, {s.x, 0}, {0, s.y}, s};
    const float wt[4] = {9.0f, 3.0f, 3.0f, 1.0f};
    V2 sum{0, 0};
    float weight = 0.0f;
    for (int k = 0; k < 4; k++) {
        I2 at{coarse.x + off[k].x, coarse.y + off[k].y};
        float r = rhoAt(X, l + 1u, at);
        if (r < 0.0f) continue;
        weight = weight + wt[k];
        if (r > 0.0f) {
            V2 p = potAt(X, l + 1u, at);
            sum.x = sum.x + wt[k] * p.x;
            sum.y = sum.y + wt[k] * p.y;
        }
    }
    float w = wmax(weight, 1e-6f);
    return V2{sum.x / w, sum.y / w};
}

// ---------------------------------------------------------------- pass drivers

double tree64(double* w, int n);

// The cells of the blocks worked on, a workgroup per block: f(wid, c, li).
template <class Fn>
void forActiveCells(Ctx& X, Fn fn) {
    uint32_t n = X.activeCount();
    for (uint32_t wid = 0; wid < n; wid++) {
        I2 b = X.activeBlock(wid);
        for (int ly = 0; ly < BLOCK; ly++)
            for (int lx = 0; lx < BLOCK; lx++) fn(wid, I2{b.x * BLOCK + lx, b.y * BLOCK + ly}, (uint32_t)(ly * BLOCK + lx));
    }
}

// ---------------------------------------------------------------- free bodies (fluid.wgsl:1181-1470)

constexpr uint32_t MAX_BODIES = WIG_MAX_BODIES, BODY_TABLE_WORDS = WIG_BODY_TABLE_WORDS;
constexpr uint32_t PUSH_P0 = 0, PUSH_X = 2, PUSH_F = 3, PUSH_SURFACE = 4, PUSH_DRAG = 5;
constexpr float EXACT_COARSE = 16777216.0f, RIGID_FIX = WIG_RIGID_FIX;
constexpr int SEEP_REACH = 128;

uint32_t bodyWord(Ctx& X, uint32_t b, uint32_t k) { return X.motion[MAX_BODIES + b * BODY_TABLE_WORDS + k]; }
float bodyF(Ctx& X, uint32_t b, uint32_t k) { return flt(bodyWord(X, b, k)); }
V2 bodyV(Ctx& X, uint32_t b, uint32_t k) { return V2{bodyF(X, b, k), bodyF(X, b, k + 1u)}; }
uint32_t liquidSlot(uint32_t b, uint32_t w) { return WIG_BODY_LIQUID_BASE + b * WIG_BODY_LIQUID_WORDS + w; }
// alive, weighed and not just found (rigidBodyOf's, cupOf's test, fluid.wgsl:1243-1246)
bool bodyInSolve(Ctx& X, uint32_t b) {
    uint32_t flags = bodyWord(X, b, WIG_BW_FLAGS);
    return !((flags & WIG_BF_ALIVE) == 0u || (flags & WIG_BF_NEW) != 0u || bodyF(X, b, WIG_BW_MASS) <= 0.0f);
}
// rigidBodyOf (fluid.wgsl:1233-1248)
uint32_t rigidBodyOf(Ctx& X, const uint32_t* v) {
    uint32_t t = wordType(v[0]);
    if (!wordHas(v[0], WIG_FL_LOOSE) || X.elem(t).kind != WIG_KIND_SOLID || X.elem(t).break_to == WIG_NO_ELEM) return NONE;
    float id = f16_value(v[3] & 0xffffu);
    if (id < 0.0f || id >= (float)MAX_BODIES) return NONE;
    uint32_t b = f2u(id);
    return bodyInSolve(X, b) ? b : NONE;
}
float rigidMass(Ctx& X, uint32_t b) { return bodyF(X, b, WIG_BW_MASS) + bodyF(X, b, WIG_BW_CARGO); }
float rigidInertia(Ctx& X, uint32_t b) { return bodyF(X, b, WIG_BW_INERTIA) + bodyF(X, b, WIG_BW_CARGO_INERTIA); }
float bodyDensity(Ctx& X, uint32_t b) { return rigidMass(X, b) / wmax((float)bodyWord(X, b, WIG_BW_CELLS), 1.0f); }
bool isHeld(Ctx& X, uint32_t b) { return (bodyWord(X, b, WIG_BW_FLAGS) & WIG_BF_HELD) != 0u; }
// wetRegionAt (fluid.wgsl:592-595)
bool wetRegionAt(Ctx& X, const uint32_t* v) {
    if (!X.motion) return false;
    uint32_t b = rigidBodyOf(X, v);
    return b != NONE && (bodyWord(X, b, WIG_BW_FLAGS) & (WIG_BF_WET | WIG_BF_HELD)) == (WIG_BF_WET | WIG_BF_HELD);
}
// bodySweptSlot, claimStep (common.wgsl:316-385): cell i's stamp of step frame
uint32_t claimStep(uint32_t frame) { return frame % WIG_CLAIM_PERIOD + 1u; }
uint32_t bodySweptSlot(Ctx& X, uint32_t i, uint32_t frame) {
    uint32_t tiles = (((uint32_t)X.W + WIG_BODY_TILE - 1u) / WIG_BODY_TILE) * (((uint32_t)X.H + WIG_BODY_TILE - 1u) / WIG_BODY_TILE);
    uint32_t base = 4u * tiles + WIG_BODY_STAT_WORDS + WIG_BODY_COUNTERS + MAX_BODIES + (2u + WIG_BODY_SUM_WORDS) * X.C;
    return base + 1u + tiles + 2u * X.C + X.C + 2u * i + (frame & 1u);
}
// cupOf, seamOf (fluid.wgsl:1252-1288): the body whose cup (seam) cell i was
// stamped last step, alive and weighed; cupBefore (fluid.wgsl:3521-3528):
// whose cup it was the step before, whatever the body's state now
uint32_t sweptBody(Ctx& X, uint32_t i, uint32_t frame, uint32_t seam) {
    if (!X.stamps || !X.motion) return NONE;
    uint32_t key = X.stamps[bodySweptSlot(X, i, frame)];
    if ((key >> 12u) != claimStep(frame) || (key & 1u) != seam) return NONE;
    uint32_t b = 2047u - ((key >> 1u) & 0x7ffu);
    return b < MAX_BODIES ? b : NONE;
}
uint32_t cupOf(Ctx& X, uint32_t i) {
    uint32_t b = sweptBody(X, i, X.P->frame - 1u, 0u);
    return b != NONE && bodyInSolve(X, b) ? b : NONE;
}
uint32_t seamOf(Ctx& X, uint32_t i) {
    uint32_t b = sweptBody(X, i, X.P->frame - 1u, 1u);
    return b != NONE && bodyInSolve(X, b) ? b : NONE;
}
uint32_t cupBefore(Ctx& X, uint32_t i) { return sweptBody(X, i, X.P->frame - 2u, 0u); }
// rigidAt, heldAt (fluid.wgsl:1422-1458): the body classify put in the drift's z
uint32_t rigidAt(Ctx& X, I2 c) {
    if (!X.motion || !X.inWorld(c)) return NONE;
    float z = X.fv(2u * X.cellIndex(c) + 1u)[2];
    uint32_t b = f2u(wmax(-z, 1.0f)) - 1u;
    return (z < 0.0f && b < MAX_BODIES) ? b : NONE;
}
uint32_t heldAt(Ctx& X, I2 c) {
    if (!X.motion || !X.inWorld(c)) return NONE;
    float z = X.fv(2u * X.cellIndex(c) + 1u)[2];
    uint32_t b = f2u(wmax(-z, 1.0f)) - 1u;
    // (a slot past the table, from a drift word classify did not write, is none)
    return (z < 0.0f && b >= MAX_BODIES && b < 2u * MAX_BODIES) ? b - MAX_BODIES : NONE;
}

// exactParts, exactCarry, exactValue (common.wgsl:1378-1412)
void exactParts(float x, float scale, uint32_t* lo, uint32_t* hi) {
    float s = rnd_even(clampf(x * scale, -9.2e18f, 9.2e18f));
    if (std::fabs(s) < 2147483648.0f) {
        int32_t v = f2i(s);
        *lo = (uint32_t)v;
        *hi = v < 0 ? 0xffffffffu : 0u;
        return;
    }
    float h = std::floor(s / 4294967296.0f);
    *lo = f2u(s - h * 4294967296.0f);
    *hi = (uint32_t)f2i(h);
}
float exactValue(uint32_t lo, uint32_t hi, float scale) {
    int32_t l = (int32_t)lo, h = (int32_t)hi;
    if ((h == 0 && l >= 0) || (h == -1 && l < 0)) return (float)l / scale;
    return ((float)h * 4294967296.0f + (float)lo) / scale;
}
// pushSlot, addPush, pushOf (fluid.wgsl:1318-1338)
uint32_t pushSlot(uint32_t b, uint32_t which, uint32_t k) { return b * WIG_BODY_PUSH_WORDS + 6u * which + 2u * k; }
void addPush(Ctx& X, uint32_t b, uint32_t which, V3 v) {
    float c[3] = {v.x, v.y, v.z};
    for (uint32_t k = 0; k < 3; k++) {
        uint32_t lo, hi;
        exactParts(c[k], EXACT_COARSE, &lo, &hi);
        uint32_t at = pushSlot(b, which, k);
        uint32_t old = X.pushes[at];
        X.pushes[at] = old + lo;
        X.pushes[at + 1u] += hi + (old + lo < old ? 1u : 0u);
    }
}
V3 pushOf(Ctx& X, uint32_t b, uint32_t which) {
    float c[3];
    for (uint32_t k = 0; k < 3; k++) {
        uint32_t at = pushSlot(b, which, k);
        c[k] = exactValue(X.pushes[at], X.pushes[at + 1u], EXACT_COARSE);
    }
    return V3{c[0], c[1], c[2]};
}
// giveWay, pushChange, pushChangeFree (fluid.wgsl:1348-1372)
V3 giveWay(Ctx& X, uint32_t b, V3 g) {
    if (bodyWord(X, b, WIG_BW_MOBILITY_AT) != X.P->frame - 1u)
        return V3{g.x / rigidMass(X, b), g.y / rigidMass(X, b), g.z / rigidInertia(X, b)};
    float m[6];
    for (uint32_t k = 0; k < 6; k++) m[k] = bodyF(X, b, WIG_BW_MOBILITY + k);
    return V3{m[0] * g.x + m[1] * g.y + m[2] * g.z, m[1] * g.x + m[3] * g.y + m[4] * g.z,
              m[2] * g.x + m[4] * g.y + m[5] * g.z};
}
V3 pushChange(Ctx& X, uint32_t b, uint32_t which) { return giveWay(X, b, pushOf(X, b, which)); }
V3 pushChangeFree(Ctx& X, uint32_t b, uint32_t which) {
    V3 g = pushOf(X, b, which);
    return V3{g.x / rigidMass(X, b), g.y / rigidMass(X, b), g.z / rigidInertia(X, b)};
}
// bodyFaceJ (fluid.wgsl:1374-1379): the face from cell c to body b's cell q
V3 bodyFaceJ(Ctx& X, I2 c, I2 q, uint32_t b) {
    V2 n{(float)(q.x - c.x), (float)(q.y - c.y)};
    V2 pos = bodyV(X, b, WIG_BW_POS);
    V2 r{(((float)c.x + 0.5f) + 0.5f * n.x) - pos.x, (((float)c.y + 0.5f) + 0.5f * n.y) - pos.y};
    return V3{n.x, n.y, r.x * n.y - r.y * n.x};
}
inline V3 scale3(V3 v, float s) { return V3{v.x * s, v.y * s, v.z * s}; }
inline V3 add3(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// addPressurePush, couplingAt (fluid.wgsl:1381-1403)
void addPressurePush(Ctx& X, I2 c, float p, uint32_t which) {
    for (int d = 0; d < 4; d++) {
        I2 q = Ctx::beside(c, d);
        uint32_t b = rigidAt(X, q);
        if (b != NONE) addPush(X, b, which, scale3(bodyFaceJ(X, c, q, b), p));
    }
}
float couplingAt(Ctx& X, I2 c, uint32_t which) {
    float sum = 0.0f;
    if (!X.motion) return sum;
    for (int d = 0; d < 4; d++) {
        I2 q = Ctx::beside(c, d);
        uint32_t b = rigidAt(X, q);
        if (b != NONE) sum = sum + dot3(bodyFaceJ(X, c, q, b), pushChange(X, b, which));
    }
    return sum;
}
// rigidVel (fluid.wgsl:1460-1465), bodyMoving (fluid.wgsl:1410-1419)
V2 rigidVel(Ctx& X, uint32_t b, V2 x) {
    V2 pos = bodyV(X, b, WIG_BW_POS);
    V2 r{x.x - pos.x, x.y - pos.y};
    float spin = bodyF(X, b, WIG_BW_SPIN);
    V2 v = bodyV(X, b, WIG_BW_VEL);
    return V2{v.x + -spin * r.y, v.y + spin * r.x};
}
V2 bodyMoving(Ctx& X, uint32_t b, V2 x, bool drag) {
    V2 pos = bodyV(X, b, WIG_BW_POS);
    V2 pull = X.pullAt(pos);
    float m = rigidMass(X, b);
    V3 ch = add3(pushChange(X, b, PUSH_SURFACE), giveWay(X, b, V3{m * pull.x, m * pull.y, 0.0f}));
    if (drag) ch = add3(ch, pushChange(X, b, PUSH_DRAG));
    V2 r{x.x - pos.x, x.y - pos.y};
    V2 rv = rigidVel(X, b, x);
    V2 px = X.pullAt(x);
    return V2{(((rv.x + px.x) - pull.x) + ch.x) + -ch.z * r.y, (((rv.y + px.y) - pull.y) + ch.y) + ch.z * r.x};
}
// bodyReach (fluid.wgsl:413-415)
float bodyReach(Ctx& X, uint32_t b, I2 n) {
    uint32_t w = bodyWord(X, b, WIG_BW_SUBCELL);
    float sx = f16_value(w & 0xffffu), sy = f16_value(w >> 16);
    return clampf(0.5f + (sx * (float)n.x + sy * (float)n.y), 0.0f, 1.0f);
}
// posedRoom (fluid.wgsl:2035-2045)
float posedRoom(Ctx& X, I2 c) {
    float room = 1.0f;
    for (int d = 0; d < 4; d++) {
        I2 q = Ctx::beside(c, d);
        uint32_t b = rigidAt(X, q);
        if (b != NONE) room = room + (0.5f - bodyReach(X, b, I2{c.x - q.x, c.y - q.y}));
    }
    return clampf(room, 0.1f, 1.9f);
}
// faceMiddle (fluid.wgsl:1473-1475)
V2 faceMiddle(I2 at, bool isU) { return isU ? V2{(float)at.x + 0.0f, (float)at.y + 0.5f} : V2{(float)at.x + 0.5f, (float)at.y + 0.0f}; }
// potentialAt (fluid.wgsl:2958-2960), the masses' potential none (binding 10 unbound)
float potentialAt(Ctx& X, V2 pos) { return X.P->earth_g * ((float)X.H - pos.y) + 0.0f; }
// seepAt (fluid.wgsl:2977-3000)
float seepAt(Ctx& X, I2 c, I2 n, uint32_t h, bool held, V2 x) {
    I2 ways[2] = {I2{-1, 0}, I2{1, 0}};
    int count = 2;
    if (n.x != 0) { ways[0] = I2{-n.x, -n.y}; count = 1; }
    int nearest = SEEP_REACH + 1;
    float p = 0.0f;
    for (int w = 0; w < count; w++) {
        for (int k = 1; k < nearest; k++) {
            I2 q{c.x + ways[w].x * k, c.y + ways[w].y * k};
            if ((held ? heldAt(X, q) : rigidAt(X, q)) == h) continue;
            V4 g = X.gridAt(q);
            if (g.z > 0.0f) {
                nearest = k;
                p = g.x + g.z * (potentialAt(X, V2{(float)q.x + 0.5f, (float)q.y + 0.5f}) - potentialAt(X, x));
            }
            break;
        }
    }
    return p;
}
// heldPush (fluid.wgsl:3007-3031)
void heldPush(Ctx& X, I2 c, uint32_t h, int32_t out[3]) {
    V2 pos = bodyV(X, h, WIG_BW_POS);
    V2 f{0.0f, 0.0f};
    float torque = 0.0f;
    for (int d = 0; d < 4; d++) {
        I2 q = Ctx::beside(c, d);
        I2 n{q.x - c.x, q.y - c.y};
        if (heldAt(X, q) == h) continue;
        V4 g = X.gridAt(q);
        V2 x{((float)c.x + 0.5f) + 0.5f * (float)n.x, ((float)c.y + 0.5f) + 0.5f * (float)n.y};
        float p = g.x;
        if (g.z > 0.0f) p = p + g.z * (potentialAt(X, V2{(float)q.x + 0.5f, (float)q.y + 0.5f}) - potentialAt(X, x));
        else if (g.z < 0.0f) p = seepAt(X, c, n, h, true, x);
        V2 push{-p * (float)n.x, -p * (float)n.y};
        f = V2{f.x + push.x, f.y + push.y};
        V2 r{x.x - pos.x, x.y - pos.y};
        torque = torque + (r.x * push.y - r.y * push.x);
    }
    out[0] = f2i(rnd_even((f.x / rigidMass(X, h)) * RIGID_FIX));
    out[1] = f2i(rnd_even((f.y / rigidMass(X, h)) * RIGID_FIX));
    out[2] = f2i(rnd_even((torque / rigidInertia(X, h)) * RIGID_FIX));
}

// sync / syncMarks (fluid.wgsl:608-659)
void pass_sync(Ctx& X, bool claims) {
    X.parts[0] = 0u;
    X.blocks[X.countSlot(COUNT_ACTIVE)] = 0u;
    X.blocks[X.countSlot(COUNT_RETIRED)] = 0u;
    X.blocks[X.countSlot(COUNT_VISCOUS)] = 0u;
    int bh = (X.H + BLOCK - 1) / BLOCK;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < (int)X.BW; bx++) {
            bool here = false, region = false;
            for (int ly = 0; ly < BLOCK; ly++)
                for (int lx = 0; lx < BLOCK; lx++) {
                    I2 c{bx * BLOCK + lx, by * BLOCK + ly};
                    if (!X.inWorld(c)) continue;
                    uint32_t i = X.cellIndex(c);
                    uint32_t* v = X.cellv(i);
                    if (X.elem(wordType(v[0])).kind == WIG_KIND_LIQUID) {
                        uint32_t home = liquidHome(v[3]);
                        if (claims && wordHas(v[0], FL_DRAWN) && home < X.C) {
                            uint32_t& d = X.gw(home, G_DEST);
                            d = wmax(d, claimOf(i));
                        }
                        here = true;
                    } else if (wetRegionAt(X, v)) {
                        region = true;
                    }
                }
            if (here) X.blocks[X.blockIndex(I2{bx, by})] |= MARK_LIQUID;
            if (region) X.blocks[X.blockIndex(I2{bx, by})] |= MARK_REGION;
        }
}

void markBlockOf(Ctx& X, V2 pos) {
    I2 b = Ctx::divI(X.cellOf(pos), BLOCK);
    if (X.inBlocks(b)) X.blocks[X.blockIndex(b)] |= MARK_LIQUID;
}

V2 pairWay(uint32_t a, uint32_t b) {
    uint32_t h = pcg(wmin(a, b) ^ pcg(wmax(a, b)));
    float angle = (float)h * (float)(6.2831853 / 4294967296.0);
    float s, c;
    sincos_own(angle, &s, &c);
    float sg = a < b ? 1.0f : -1.0f;
    return V2{c * sg, s * sg};
}

// apart (fluid.wgsl:713-734)
V2 apart(Ctx& X, uint32_t k, uint32_t h, V2 pos, uint32_t id) {
    uint32_t start = X.gw(h, G_START), n = X.gw(h, G_SORT);
    if (n < 2u) return pos;
    int32_t px = 0, py = 0;
    for (uint32_t m = start; m < start + n && m < X.cap; m++) {
        if (m == k) continue;
        uint32_t* o = X.item(X.sorted, m);
        V2 d{pos.x - flt(o[0]), pos.y - flt(o[1])};
        float l = std::sqrt(d.x * d.x + d.y * d.y);
        if (l < APART) {
            V2 way = l == 0.0f ? pairWay(id, X.item(X.sorted, X.cap + m)[2]) : V2{d.x / l, d.y / l};
            float s = 0.5f * (APART - l) * APART_FIX;
            px = (int32_t)((uint32_t)px + (uint32_t)f2i(rnd_even(s * way.x)));
            py = (int32_t)((uint32_t)py + (uint32_t)f2i(rnd_even(s * way.y)));
        }
    }
    float cx = std::floor(pos.x), cy = std::floor(pos.y);
    V2 to{pos.x + (float)px / APART_FIX, pos.y + (float)py / APART_FIX};
    V2 r;
    r.x = (to.x >= cx + APART && to.x <= cx + 1.0f - APART) ? to.x : pos.x;
    r.y = (to.y >= cy + APART && to.y <= cy + 1.0f - APART) ? to.y : pos.y;
    return r;
}

// rankById (fluid.wgsl:668-678)
uint32_t rankById(Ctx& X, uint32_t h, uint32_t k, uint32_t id, uint32_t word, uint32_t drawn) {
    uint32_t start = X.gw(h, G_START);
    uint32_t mine = wordType(word) == drawn ? 1u : 0u;
    uint32_t r = 0;
    for (uint32_t m = start; m < start + X.gw(h, G_SORT) && m < X.cap; m++) {
        uint32_t* other = X.item(X.sorted, X.cap + m);
        uint32_t theirs = wordType(other[0]) == drawn ? 1u : 0u;
        r += (theirs < mine || (theirs == mine && (other[2] < id || (other[2] == id && m < k)))) ? 1u : 0u;
    }
    return r;
}

// sharedLife (fluid.wgsl:4149-4161)
uint32_t sharedLife(Ctx& X, uint32_t life, uint32_t was, uint32_t now, uint32_t id) {
    if (now == was) return life;
    float l = (float)life;
    if (now < was) l = l * (float)now / (float)was;
    else l = 255.0f - (255.0f - l) * (255.0f - (float)now) / (255.0f - (float)was);
    X.seedRng(id, X.P->frame, X.P->seed ^ 0x5a17u);
    return wmin(f2u(std::floor(l + X.rnd())), 255u);
}

// syncParticles (fluid.wgsl:767-831); parts filled in sorted's order.
void pass_syncParticles(Ctx& X) {
    uint32_t live = wmin(X.sorted[0], X.cap);
    for (uint32_t k = 0; k < live; k++) {
        bool keep = false;
        Particle q = X.toParticle(X.sorted, k);
        uint32_t h = X.cellIndex(X.cellOf(q.pos));
        q.pos = apart(X, k, h, q.pos, q.id);
        uint32_t d = X.gw(h, G_DEST);
        if (d == DEST_KEEP) {
            keep = true;
            markBlockOf(X, q.pos);
        } else if ((d & DEST_ASIDE) != 0u && (d & ~DEST_ASIDE) < X.C) {
            uint32_t to = d & ~DEST_ASIDE;
            // not into another body's cup (fluid.wgsl:785-793)
            if (cupOf(X, to) == NONE)
                q.pos = V2{(float)(to % (uint32_t)X.W) + (q.pos.x - std::floor(q.pos.x)),
                           (float)(to / (uint32_t)X.W) + (q.pos.y - std::floor(q.pos.y))};
            keep = true;
            markBlockOf(X, q.pos);
        } else if (isClaim(d) && claimedCell(d) < X.C) {
            uint32_t to = claimedCell(d);
            uint32_t* v = X.cellv(to);
            uint32_t n = liquidCount(v[3]);
            if (n == LIQUID_COUNT_MAX || X.gw(h, G_SORT) <= n || rankById(X, h, k, q.id, q.word, wordType(v[0])) < n) {
                if (to != h) {
                    q.pos = V2{(float)(to % (uint32_t)X.W) + (q.pos.x - std::floor(q.pos.x)),
                               (float)(to / (uint32_t)X.W) + (q.pos.y - std::floor(q.pos.y))};
                }
                q.temp = Ctx::cellTemp(v);
                uint32_t drawn = X.gw(h, G_TYPE);
                uint32_t pt = wordType(q.word);
                if (holdsSolute(pt) && pt == (drawn & 0xffu) && wordType(v[0]) == pt &&
                    (wordAux(q.word) == ((drawn >> 8u) & 0xffu) || wordAux(q.word) == 0u)) {
                    uint32_t life = sharedLife(X, wordAux(q.word) == 0u ? 0u : wordLife(q.word), (drawn >> 16u) & 0xffu,
                                               wordLife(v[0]), q.id);
                    uint32_t w = wordWithout(v[0], FL_DRAWN);
                    uint32_t solute = wordAux(w) != 0u ? wordAux(w) : ((drawn >> 8u) & 0xffu);
                    q.word = packWord(pt, life > 0u ? solute : 0u, life, wordShade(w), wordFlags(w));
                } else if (drawnAs(q.word) == (drawn & 0xffffu)) {
                    q.word = wordWithout(v[0], FL_DRAWN);
                }
                keep = true;
            }
        }
        if (keep) {
            uint32_t m = X.parts[0]++;
            if (m < X.cap) X.storeParticle(m, q);
        }
    }
}

// seedId, seedPos (fluid.wgsl:835-855)
uint32_t seedId(Ctx& X, I2 c, uint32_t j) {
    uint32_t h = (((uint32_t)c.y * (uint32_t)X.W + (uint32_t)c.x) * 0x9e3779b9u) ^ (X.P->frame * 0x85ebca6bu) ^ (j * 0xc2b2ae35u);
    h ^= h >> 16u;
    h *= 0x7feb352du;
    h ^= h >> 15u;
    return h;
}
V2 seedPos(Ctx& X, I2 c, uint32_t j, uint32_t n) {
    if (n == 1u) return V2{(float)c.x + 0.5f, (float)c.y + 0.5f};
    float rx = X.rnd();
    float ry = X.rnd();
    V2 r{rx - 0.5f, ry - 0.5f};
    if (n <= 4u) {
        static const float qx[4] = {0.0f, 1.0f, 1.0f, 0.0f}, qy[4] = {0.0f, 1.0f, 0.0f, 1.0f};
        return V2{(float)c.x + 0.25f + 0.5f * qx[j] + 0.3f * r.x, (float)c.y + 0.25f + 0.5f * qy[j] + 0.3f * r.y};
    }
    return V2{(float)c.x + 0.5f + 0.9f * r.x, (float)c.y + 0.5f + 0.9f * r.y};
}

// syncSeed (fluid.wgsl:863-890); cells in row order.
void pass_syncSeed(Ctx& X) {
    for (int y = 0; y < X.H; y++)
        for (int x = 0; x < X.W; x++) {
            I2 c{x, y};
            uint32_t i = X.cellIndex(c);
            uint32_t* v = X.cellv(i);
            if (X.elem(wordType(v[0])).kind != WIG_KIND_LIQUID) continue;
            uint32_t home = liquidHome(v[3]);
            uint32_t want = liquidCount(v[3]);
            uint32_t n = 0;
            if (!wordHas(v[0], FL_DRAWN)) {
                n = X.ppc;
            } else if (home >= X.C || X.gw(home, G_DEST) != claimOf(i)) {
                n = wmax(want, 1u);
            } else if (want > X.gw(home, G_SORT) && want < LIQUID_COUNT_MAX) {
                n = want - X.gw(home, G_SORT);
            }
            X.seedRng(i, X.P->frame, X.P->seed ^ 0x5eedu);
            if (n == 0u) continue;
            uint32_t m = X.parts[0];
            X.parts[0] += n;
            for (uint32_t j = 0; j < n; j++) {
                Particle q;
                q.pos = seedPos(X, c, j, n);
                q.vel = Ctx::cellVel(v);
                q.word = wordWithout(v[0], FL_DRAWN);
                q.temp = Ctx::cellTemp(v);
                q.id = seedId(X, c, j);
                q.affine = V4{0, 0, 0, 0};
                if (m + j < X.cap) X.storeParticle(m + j, q);
            }
        }
}

// compact (fluid.wgsl:896-921); the list in block-index order.
void pass_compact(Ctx& X) {
    int bh = (int)(X.B / X.BW);
    std::vector<uint32_t> marks(X.blocks, X.blocks + X.B);
    for (uint32_t n = 0; n < X.B; n++) {
        I2 b{(int)(n % X.BW), (int)(n / X.BW)};
        uint32_t m = 0;
        for (int y = -1; y <= 1; y++)
            for (int x = -1; x <= 1; x++) {
                I2 o{b.x + x, b.y + y};
                if (X.inBlocks(o)) m |= marks[X.blockIndex(o)];
            }
        (void)bh;
        bool near = (m & MARK_LIQUID) != 0u;
        bool liquid = (m & (MARK_LIQUID | MARK_REGION)) != 0u;
        bool was = (X.blocks[X.stateSlot(n)] & ACTIVE) != 0u;
        X.blocks[X.stateSlot(n)] = (liquid ? ACTIVE : 0u) | (near ? NEAR_LIQUID : 0u);
        if (liquid) X.blocks[X.activeSlot(X.blocks[X.countSlot(COUNT_ACTIVE)]++)] = n;
        else if (was) X.blocks[X.retiredSlot(X.blocks[X.countSlot(COUNT_RETIRED)]++)] = n;
    }
}

void clearCell(Ctx& X, uint32_t i) {
    for (uint32_t g = 0; g < CELL_WORDS; g++) X.gw(i, g) = 0u;
}

// retire (fluid.wgsl:924-951)
void pass_retire(Ctx& X) {
    uint32_t nr = X.blocks[X.countSlot(COUNT_RETIRED)];
    for (uint32_t wid = 0; wid < nr; wid++) {
        uint32_t n = X.blocks[X.retiredSlot(wid)];
        for (int ly = 0; ly < BLOCK; ly++)
            for (int lx = 0; lx < BLOCK; lx++) {
                I2 c{(int)(n % X.BW) * BLOCK + lx, (int)(n / X.BW) * BLOCK + ly};
                if (!X.inWorld(c)) continue;
                uint32_t i = X.cellIndex(c);
                std::memset(X.fv(2u * i), 0, 32);
                clearCell(X, i);
                int fs[4][3];
                X.facesOf(c, fs);
                for (int j = 0; j < 4; j++) {
                    if (fs[j][2] < 0) continue;
                    uint32_t f = X.faceIndex(I2{fs[j][0], fs[j][1]}, fs[j][2] == 1);
                    std::memset(X.fv(X.faceSlot(f)), 0, 16);
                    X.viscLast(f) = 0.0f;
                    X.counters[X.sumSlot(f)] = 0u;
                    X.counters[X.sumSlot(f) + 1u] = 0u;
                }
                if (lx == 0 && ly == 0) X.blocks[n] = 0u;
            }
    }
}

// clear (fluid.wgsl:962-985)
void pass_clear(Ctx& X) {
    uint32_t na = X.activeCount();
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        X.blocks[X.blockIndex(b)] = 0u;
        for (int ly = 0; ly < BLOCK; ly++)
            for (int lx = 0; lx < BLOCK; lx++) {
                I2 c{b.x * BLOCK + lx, b.y * BLOCK + ly};
                if (!X.inWorld(c)) continue;
                uint32_t i = X.cellIndex(c);
                clearCell(X, i);
                X.gw(i, G_REGION) = i;
                int fs[4][3];
                X.facesOf(c, fs);
                for (int j = 0; j < 4; j++) {
                    if (fs[j][2] < 0) continue;
                    uint32_t f = X.faceIndex(I2{fs[j][0], fs[j][1]}, fs[j][2] == 1);
                    X.counters[X.sumSlot(f)] = 0u;
                    X.counters[X.sumSlot(f) + 1u] = 0u;
                }
            }
    }
}

// splatAxis (fluid.wgsl:1000-1015)
void splatAxis(Ctx& X, V2 s, float vel, V2 g, bool isU) {
    float fx0 = std::floor(s.x), fy0 = std::floor(s.y);
    I2 b{f2i(fx0), f2i(fy0)};
    V2 f{s.x - fx0, s.y - fy0};
    for (int j = 0; j < 4; j++) {
        int ox = j & 1, oy = j >> 1;
        float w = (ox == 1 ? f.x : 1.0f - f.x) * (oy == 1 ? f.y : 1.0f - f.y);
        I2 at{b.x + ox, b.y + oy};
        if (w <= 0.0f || !X.faceInWorld(at, isU)) continue;
        uint32_t slot = X.sumSlot(X.faceIndex(at, isU));
        float there = vel + (g.x * ((float)at.x - s.x) + g.y * ((float)at.y - s.y));
        X.counters[slot] += (uint32_t)f2i(rnd_even(there * w * FIX));
        X.counters[slot + 1u] += (uint32_t)f2i(rnd_even(w * FIX));
    }
}

bool walls(Ctx& X, I2 c) {
    if (!X.inWorld(c)) return true;
    uint32_t k = X.kindOfCell(X.cellIndex(c));
    return k == WIG_KIND_SOLID || k == WIG_KIND_POWDER;
}

// splatDensity (fluid.wgsl:1069-1087)
void splatDensity(Ctx& X, V2 pos, float room) {
    V2 s{pos.x - 0.5f, pos.y - 0.5f};
    float fx0 = std::floor(s.x), fy0 = std::floor(s.y);
    I2 b{f2i(fx0), f2i(fy0)};
    V2 f{s.x - fx0, s.y - fy0};
    for (int j = 0; j < 4; j++) {
        int ox = j & 1, oy = j >> 1;
        float w = (ox == 1 ? f.x : 1.0f - f.x) * (oy == 1 ? f.y : 1.0f - f.y);
        I2 at{b.x + ox, b.y + oy};
        if (walls(X, at)) {
            I2 x{b.x + 1 - ox, at.y};
            I2 y{at.x, b.y + 1 - oy};
            I2 xy{b.x + 1 - ox, b.y + 1 - oy};
            if (!walls(X, x)) at = x;
            else if (!walls(X, y)) at = y;
            else if (!walls(X, xy)) at = xy;
            else at = I2{-1, -1};
        }
        if (X.inWorld(at) && w > 0.0f) X.gw(X.cellIndex(at), G_DENSITY) += f2u(rnd_even(w * room * FIX));
    }
}

// gather (fluid.wgsl:1017-1039), the air's push left out (no air bound).
void pass_gather(Ctx& X) {
    uint32_t live = X.partsLive();
    for (uint32_t k = 0; k < live; k++) {
        Particle q = X.toParticle(X.parts, k);
        splatAxis(X, V2{q.pos.x - 0.0f, q.pos.y - 0.5f}, q.vel.x, V2{q.affine.x, q.affine.y}, true);
        splatAxis(X, V2{q.pos.x - 0.5f, q.pos.y - 0.0f}, q.vel.y, V2{q.affine.z, q.affine.w}, false);
        uint32_t home = X.cellIndex(X.cellOf(q.pos));
        X.gw(home, G_COUNT) += 1u;
        X.gw(home, G_MASS) += f2u(rnd_even(X.liquidDensity(q.word, q.temp) * FIX));
        splatDensity(X, q.pos, X.liquidVolume(q.word, q.temp));
    }
}

bool mayBeSealed(Ctx& X, I2 c) {
    if (countAt(X, c) != 0) return false;
    uint32_t i = X.cellIndex(c);
    return X.fv(2u * i)[2] > 0.0f || X.fv(2u * i + 1u)[2] != 0.0f;
}
bool wasOpen(Ctx& X, I2 q) {
    if (!X.inWorld(q) || countAt(X, q) < 0) return false;
    uint32_t sb = 1u << ((X.P->frame + 1u) & 1u);
    return (f2u(X.fv(2u * X.cellIndex(q) + 1u)[3]) & sb) == 0u;
}

// sealJoin, sealAnchor (fluid.wgsl:1531-1554)
void pass_sealJoin(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c) || !mayBeSealed(X, c)) return;
        for (int d = 0; d < 2; d++) {
            I2 n = d == 0 ? I2{c.x + 1, c.y} : I2{c.x, c.y + 1};
            if (mayBeSealed(X, n)) ufJoin(X, X.cellIndex(c), X.cellIndex(n));
        }
    });
}
void pass_sealAnchor(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c) || !mayBeSealed(X, c)) return;
        if (wasOpen(X, Ctx::beside(c, 0)) || wasOpen(X, Ctx::beside(c, 1)) || wasOpen(X, Ctx::beside(c, 2)) ||
            wasOpen(X, Ctx::beside(c, 3)))
            X.gw(ufFind(X, X.cellIndex(c)), G_REGION) |= REGION_OPEN;
    });
}

// columnWeight (fluid.wgsl:1566-1575)
float columnWeight(Ctx& X, I2 p, float density) {
    int over = 0;
    I2 q{p.x, p.y - 1};
    while (over < COLUMN_MOST && countAt(X, q) > 0) {
        over += 1;
        q.y -= 1;
    }
    return density * X.P->earth_g * ((float)over + 0.5f);
}

// classify (fluid.wgsl:1578-1696)
void pass_classify(Ctx& X) {
    uint32_t na = X.activeCount();
    uint32_t mine = 1u << (X.P->frame & 1u);
    uint32_t fall0 = 4u << (X.P->frame & 1u);
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        uint32_t blockBits = 0;
        for (int ly = 0; ly < BLOCK; ly++)
            for (int lx = 0; lx < BLOCK; lx++) {
                I2 p{b.x * BLOCK + lx, b.y * BLOCK + ly};
                if (!X.inWorld(p)) continue;
                uint32_t i = X.cellIndex(p);
                int n = countAt(X, p);
                V4 c{0, 0, 0, 0};
                float* wasp = X.fv(2u * i);
                float* wdp = X.fv(2u * i + 1u);
                V4 was{wasp[0], wasp[1], wasp[2], wasp[3]};
                V4 wasDrift{wdp[0], wdp[1], wdp[2], wdp[3]};
                bool sealed = false;
                if (n == 0 && mayBeSealed(X, p)) sealed = (ufLink(X, ufFind(X, i)) & REGION_OPEN) == 0u;
                uint32_t rigid = NONE, held = NONE;
                uint32_t seam = n < 0 ? NONE : seamOf(X, i);
                if (seam != NONE) {
                    // a gap the stamp opened in a body's wall: the body's (fluid.wgsl:1604-1613)
                    c.z = -1.0f;
                    rigid = seam;
                    if (isHeld(X, seam)) { held = seam; rigid = NONE; }
                    sealed = false;
                } else if (n < 0) {
                    c.z = -1.0f;
                    // a free body's cell, or powder in its cup, its cargo (fluid.wgsl:1614-1627)
                    if (X.motion) {
                        rigid = rigidBodyOf(X, X.cellv(i));
                        if (rigid == NONE && X.kindOfCell(i) == WIG_KIND_POWDER) rigid = cupOf(X, i);
                    }
                    if (rigid != NONE && isHeld(X, rigid)) { held = rigid; rigid = NONE; }
                } else if (n > 0) {
                    V2 li = liquidIn(X, i);
                    c = V4{0, 0, li.x, li.y};
                } else {
                    float fluid = 0.0f, wallsN = 0.0f;
                    V2 mean{0, 0};
                    for (int d = 0; d < 4; d++) {
                        I2 q = Ctx::beside(p, d);
                        int m = countAt(X, q);
                        if (m < 0) wallsN = wallsN + 1.0f;
                        else if (m > 0) {
                            fluid = fluid + 1.0f;
                            V2 li = liquidIn(X, X.cellIndex(q));
                            mean.x = mean.x + li.x;
                            mean.y = mean.y + li.y;
                        }
                    }
                    if (fluid >= 2.0f && fluid + wallsN >= 3.0f) {
                        c = V4{0, 0, mean.x / fluid, mean.y / fluid};
                    } else if (sealed) {
                        c = fluid > 0.0f ? V4{0, 0, mean.x / fluid, mean.y / fluid} : V4{0, 0, 1.0f, 0.0f};
                    }
                }
                uint32_t liquid = (c.z > 0.0f || rigid != NONE || held != NONE) ? mine : 0u;
                V4 drift{0.0f, 0.0f, sealed ? 1.0f : 0.0f, (float)((f2u(wasDrift.w) & ~(mine | fall0)) | liquid)};
                if (rigid != NONE) drift.z = -1.0f - (float)rigid;
                else if (held != NONE) drift.z = -1.0f - (float)(held + MAX_BODIES);
                if (c.z > 0.0f) {
                    if (was.z > 0.0f) {
                        c.x = was.x;
                        drift.x = wasDrift.x * DRIFT_KEEP;
                    } else {
                        c.x = columnWeight(X, p, c.z);
                    }
                    blockBits |= c.w > 0.0f ? (HAS_FLUID | HAS_VISCOUS) : HAS_FLUID;
                }
                wasp[0] = c.x; wasp[1] = c.y; wasp[2] = c.z; wasp[3] = c.w;
                wdp[0] = drift.x; wdp[1] = drift.y; wdp[2] = drift.z; wdp[3] = drift.w;
            }
        X.blocks[X.stateSlot(X.blockIndex(b))] |= blockBits;
        if (blockBits & HAS_VISCOUS) X.blocks[X.countSlot(COUNT_VISCOUS)] = 1u;
    }
}

float obstacleVelAxis(Ctx& X, I2 c, int axis) {
    if (!X.inWorld(c)) return 0.0f;
    uint32_t* v = X.cellv(X.cellIndex(c));
    uint32_t k = X.elem(wordType(v[0])).kind;
    if (k == WIG_KIND_SOLID || k == WIG_KIND_GAS) return 0.0f;
    V2 cv = Ctx::cellVel(v);
    return (axis == 0 ? cv.x : cv.y) * POWDER_PUSH;
}

// faceViscosity, lastPush, wasLiquid (fluid.wgsl:3279-3317)
float faceViscosity(V4 ga, V4 gb) {
    if (ga.z < 0.0f || gb.z < 0.0f) return 0.0f;
    float fa = ga.z > 0.0f ? 1.0f : 0.0f, fb = gb.z > 0.0f ? 1.0f : 0.0f;
    return (fa * ga.w + fb * gb.w) / wmax(fa + fb, 1.0f);
}
bool wasLiquid(Ctx& X, I2 c) {
    uint32_t sb = 1u << ((X.P->frame + 1u) & 1u);
    return (f2u(X.fv(2u * X.cellIndex(c) + 1u)[3]) & sb) != 0u;
}
float lastPush(Ctx& X, I2 a, I2 at, V4 ga, V4 gb) {
    if ((ga.z > 0.0f && !wasLiquid(X, a)) || (gb.z > 0.0f && !wasLiquid(X, at))) return 0.0f;
    return fineBeta(ga.z, gb.z, X.shareAt(a), X.shareAt(at)) * (gb.x - ga.x);
}

// setBodyFace (fluid.wgsl:1840-1859)
void setBodyFace(Ctx& X, uint32_t f, I2 at, bool isU, V4 ga, V4 gb, uint32_t ra, uint32_t rb, bool drag) {
    V2 x = faceMiddle(at, isU);
    float now = 0.0f, u = 0.0f;
    if (ra != NONE && rb != NONE) {
        V2 ma = bodyMoving(X, ra, x, drag), mb = bodyMoving(X, rb, x, drag);
        V2 va = rigidVel(X, ra, x), vb = rigidVel(X, rb, x);
        now = 0.5f * (isU ? ma.x + mb.x : ma.y + mb.y);
        u = 0.5f * (isU ? va.x + vb.x : va.y + vb.y);
    } else {
        uint32_t b = ra != NONE ? ra : rb;
        V2 m = bodyMoving(X, b, x, drag), v = rigidVel(X, b, x);
        now = isU ? m.x : m.y;
        u = isU ? v.x : v.y;
    }
    V4 other = ra != NONE ? gb : ga;
    float nu = ((ra == NONE || rb == NONE) && other.z > 0.0f) ? other.w : 0.0f;
    float* fp = X.fv(X.faceSlot(f));
    fp[0] = now; fp[1] = u; fp[2] = 1.0f; fp[3] = nu;
    X.viscRhs(f) = now;
}

// setFace (fluid.wgsl:1936-1980), the wind's drag none (no air bound).
void setFace(Ctx& X, I2 at, bool isU) {
    uint32_t f = X.faceIndex(at, isU);
    I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
    int axis = isU ? 0 : 1;
    V4 ga = X.gridAt(a), gb = X.gridAt(at);
    uint32_t ra = rigidAt(X, a), rb = rigidAt(X, at);
    if (ra != NONE || rb != NONE) {
        setBodyFace(X, f, at, isU, ga, gb, ra, rb, false);
        return;
    }
    uint32_t slot = X.sumSlot(f);
    int32_t weight = (int32_t)X.counters[slot + 1u];
    float u = 0.0f, held = 0.0f;
    if (ga.z < 0.0f && gb.z < 0.0f) {
        held = -1.0f;
    } else if (ga.z < 0.0f || gb.z < 0.0f) {
        u = obstacleVelAxis(X, ga.z < 0.0f ? a : at, axis);
        held = 1.0f;
    } else if (weight > 0) {
        u = (float)(int32_t)X.counters[slot] / (float)weight;
        held = 1.0f;
    }
    float now = u;
    if (held > 0.0f && ga.z >= 0.0f && gb.z >= 0.0f) {
        V2 pull = X.pullAt(V2{0, 0});
        now = now + (isU ? pull.x : pull.y);
    }
    float start = now;
    float fvisc = faceViscosity(ga, gb);
    if (fvisc > 0.0f) {
        now = now - lastPush(X, a, at, ga, gb);
        start = now + X.viscLast(f);
    }
    float* fp = X.fv(X.faceSlot(f));
    fp[0] = start; fp[1] = u; fp[2] = held; fp[3] = fvisc;
    X.viscRhs(f) = now;
}

void pass_setFaces(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        int fs[4][3];
        X.facesOf(c, fs);
        for (int j = 0; j < 4; j++)
            if (fs[j][2] >= 0) setFace(X, I2{fs[j][0], fs[j][1]}, fs[j][2] == 1);
    });
}

// viscousFace (fluid.wgsl:3347-3403)
void viscousFace(Ctx& X, I2 at, bool isU, int color) {
    if (((at.x + at.y) & 1) != color) return;
    I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
    V4 ga = X.gridAt(a), gb = X.gridAt(at);
    uint32_t ra = rigidAt(X, a), rb = rigidAt(X, at);
    bool surface = (ra != NONE) != (rb != NONE) && (ra != NONE ? gb.z : ga.z) > 0.0f;
    if (!surface && (ga.z < 0.0f || gb.z < 0.0f || ra != NONE || rb != NONE)) return;
    uint32_t fi = X.faceIndex(at, isU);
    float* fp = X.fv(X.faceSlot(fi));
    float nu = fp[3];
    if (nu <= 0.0f) return;
    float heavy = 1.0f;
    if (surface) {
        float liquid = ra != NONE ? gb.z : ga.z;
        heavy = 2.0f * liquid / (liquid + bodyDensity(X, ra != NONE ? ra : rb));
    }
    V2 through{ga.z > 0.0f ? ga.w : 0.0f, gb.z > 0.0f ? gb.w : 0.0f};
    float sum = 0.0f, n = 0.0f;
    for (int d = 0; d < 4; d++) {
        I2 o = Ctx::beside(at, d);
        bool across = isU == (d >= 2);
        V4 other{0, 0, -1.0f, 0};
        if (X.faceInWorld(o, isU)) {
            float* op = X.fv(X.faceSlot(X.faceIndex(o, isU)));
            other = V4{op[0], op[1], op[2], op[3]};
        }
        float k = (d & 1) == 1 ? through.y : through.x;
        if (across) k = other.z < 0.0f ? nu : 2.0f * nu * other.w / wmax(nu + other.w, 1e-12f);
        if (other.z < 0.0f) n = n + k * (across ? 2.0f : 1.0f);
        else if (other.z > 0.0f) { sum = sum + k * other.x; n = n + k; }
    }
    fp[0] = mixf(fp[0], (X.viscRhs(fi) + heavy * sum) / (1.0f + heavy * n), VISC_OMEGA);
}

// viscosityRed/Black/unpress (fluid.wgsl:3409-3466)
void pass_viscosity(Ctx& X, int color) {
    uint32_t na = X.activeCount();
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        if ((X.statesOf(I2{b.x - 1, b.y - 1}, I2{b.x + 1, b.y + 1}) & HAS_VISCOUS) == 0u) continue;
        for (int ly = 0; ly < BLOCK; ly++)
            for (int lx = 0; lx < BLOCK; lx++) {
                I2 c{b.x * BLOCK + lx, b.y * BLOCK + ly};
                if (!X.inWorld(c)) continue;
                int fs[4][3];
                X.facesOf(c, fs);
                for (int j = 0; j < 4; j++) {
                    if (fs[j][2] < 0) continue;
                    I2 at{fs[j][0], fs[j][1]};
                    bool isU = fs[j][2] == 1;
                    if (color < 2) { viscousFace(X, at, isU, color); continue; }
                    I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
                    V4 ga = X.gridAt(a), gb = X.gridAt(at);
                    uint32_t fi = X.faceIndex(at, isU);
                    if (rigidAt(X, a) == NONE && rigidAt(X, at) == NONE && faceViscosity(ga, gb) > 0.0f) {
                        float* fp = X.fv(X.faceSlot(fi));
                        X.viscLast(fi) = fp[0] - X.viscRhs(fi);
                        fp[0] = fp[0] + lastPush(X, a, at, ga, gb);
                    } else if (X.viscLast(fi) != 0.0f) {
                        X.viscLast(fi) = 0.0f;
                    }
                }
            }
    }
}

// divergence (fluid.wgsl:1996-2025)
void pass_divergence(Ctx& X) {
    X.blocks[X.countSlot(COUNT_RESIDUAL)] = 0u;
    X.blocks[X.countSlot(COUNT_CYCLES)] = 0u;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        if (X.fv(2u * i)[2] <= 0.0f) return;
        float out = X.fv(X.faceSlot(X.uFace(c.x + 1, c.y)))[0] - X.fv(X.faceSlot(X.uFace(c.x, c.y)))[0] +
                    X.fv(X.faceSlot(X.vFace(c.x, c.y + 1)))[0] - X.fv(X.faceSlot(X.vFace(c.x, c.y)))[0];
        X.fv(2u * i)[1] = out;
        float n = X.densityAt(c);
        float room = posedRoom(X, c);
        X.fv(2u * i + 1u)[1] = X.fv(2u * i + 1u)[2] < 0.0f ? 0.0f : -SPREAD * (n - room);
    });
}

// cgStart .. cgPrepare (fluid.wgsl:2665-2732)
void pass_cgStart(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        float* g = X.cg + 4u * (size_t)i;
        g[0] = X.gridAt(c).x; g[1] = 0; g[2] = 0; g[3] = 0;
        X.gw(i, G_REGION) = i;
    });
}
void pass_cgJoin(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c) || X.gridAt(c).z <= 0.0f) return;
        for (int d = 0; d < 2; d++) {
            I2 n = d == 0 ? I2{c.x + 1, c.y} : I2{c.x, c.y + 1};
            if (rhoAt(X, 0, n) > 0.0f) ufJoin(X, X.cellIndex(c), X.cellIndex(n));
        }
    });
}
void pass_cgAnchor(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c) || X.gridAt(c).z <= 0.0f) return;
        for (int d = 0; d < 4; d++) {
            I2 n = Ctx::beside(c, d);
            if (X.inWorld(n) && rhoAt(X, 0, n) == 0.0f) {
                X.gw(ufFind(X, X.cellIndex(c)), G_REGION) |= REGION_OPEN;
                return;
            }
        }
    });
}
// The squared norm of v over the active blocks, in the blocks' tree order
// (64-cell trees into per-block partials, then sumBlocks' order).
std::vector<double> g_norm64;
template <class Fn>
double norm2Blocks(Ctx& X, Fn value) {
    g_norm64.assign(2u * X.B, 0.0);
    uint32_t na = X.activeCount();
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        double w[64];
        for (int li = 0; li < 64; li++) {
            I2 c{b.x * BLOCK + li % BLOCK, b.y * BLOCK + li / BLOCK};
            double v = X.inWorld(c) ? value(c) : 0.0;
            w[li] = v * v;
        }
        g_norm64[2u * X.blockIndex(b)] = tree64(w, 64);
    }
    double w[256];
    for (uint32_t li = 0; li < 256; li++) {
        double s = 0.0;
        for (uint32_t k = li; k < X.B; k += 256u)
            if ((X.blocks[X.stateSlot(k)] & ACTIVE) != 0u) s = s + g_norm64[2u * k];
        w[li] = s;
    }
    return tree64(w, 256);
}

void pass_cgResidual(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        if (X.gridAt(c).z > 0.0f) X.cg[4u * (size_t)X.cellIndex(c) + 1u] = -residualAt(X, 0, c).x - couplingAt(X, c, PUSH_X);
    });
    X.bnorm2 = norm2Blocks(X, [&](I2 c) -> double {
        uint32_t i = X.cellIndex(c);
        return X.fv(2u * i)[2] > 0.0f ? (double)X.fv(2u * i)[1] : 0.0;
    });
}
void pass_cgPrepare(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        X.fv(2u * i)[0] = 0.0f;
        if (X.fv(2u * i)[2] > 0.0f) X.fv(2u * i)[1] = -X.cg[4u * (size_t)i + 1u];
    });
}

// relaxRims, relaxTile (fluid.wgsl:2096-2182)
void pass_relaxRims(Ctx& X) {
    if (X.converged()) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        if (X.fv(2u * i)[2] > 0.0f) {
            X.gw(i, G_RIM) = bits(X.fv(2u * i)[0]);
            X.gw(i, G_RIM + 1u) = bits(X.fv(2u * i + 1u)[0]);
        }
    });
}

I2 tileBlock(Ctx& X, uint32_t wid, int shift) {
    if (wid < X.activeCount()) return X.activeBlock(wid);
    int wide = (int)X.BW, high = (int)(X.B / X.BW);
    int j = (int)wid - (int)X.B;
    if (shift == 0 || j < 0 || j > high + wide) return I2{-1, -1};
    return j <= high ? I2{wide, j} : I2{j - high - 1, high};
}

void relaxTile(Ctx& X, uint32_t wid, int shift) {
    I2 b = tileBlock(X, wid, shift);
    I2 origin{b.x * BLOCK - shift, b.y * BLOCK - shift};
    uint32_t live = 0;
    if (b.x >= 0 && origin.x < X.W && origin.y < X.H && !X.converged())
        live = X.statesOf(Ctx::divI(origin, BLOCK), Ctx::divI(I2{origin.x + BLOCK - 1, origin.y + BLOCK - 1}, BLOCK)) & HAS_FLUID;
    if (live == 0u) return;
    V2 pot[RIM * RIM];
    float trho[RIM * RIM], tshare[RIM * RIM];
    for (int k = 0; k < RIM * RIM; k++) {
        I2 c{origin.x - 1 + k % RIM, origin.y - 1 + k / RIM};
        V2 p{0, 0};
        float rho = -1.0f;
        if (X.inWorld(c)) {
            uint32_t j = 2u * X.cellIndex(c);
            p = V2{X.fv(j)[0], X.fv(j + 1u)[0]};
            rho = X.fv(j)[2];
            if (rho > 0.0f) {
                uint32_t i = X.cellIndex(c);
                p = V2{flt(X.gw(i, G_RIM)), flt(X.gw(i, G_RIM + 1u))};
            }
        }
        pot[k] = p;
        trho[k] = rho;
        tshare[k] = X.shareAt(c);
    }
    struct T { V2 rhs; float bx, by, bz, bw, dx, dy, diag; bool solving; int color, t; uint32_t idx; };
    T th[64];
    for (int ly = 0; ly < BLOCK; ly++)
        for (int lx = 0; lx < BLOCK; lx++) {
            T& s = th[ly * BLOCK + lx];
            I2 me{origin.x + lx, origin.y + ly};
            int t = (ly + 1) * RIM + lx + 1;
            float rho = trho[t];
            s.rhs = V2{0, 0};
            s.bx = s.by = s.bz = s.bw = 0.0f;
            s.idx = 0;
            if (rho > 0.0f) {
                uint32_t i = 2u * X.cellIndex(me);
                s.rhs = V2{X.fv(i)[1], X.fv(i + 1u)[1]};
                float d = tshare[t];
                s.bx = fineBeta(rho, trho[t - 1], d, tshare[t - 1]);
                s.by = fineBeta(rho, trho[t + 1], d, tshare[t + 1]);
                s.bz = fineBeta(rho, trho[t - RIM], d, tshare[t - RIM]);
                s.bw = fineBeta(rho, trho[t + RIM], d, tshare[t + RIM]);
                s.idx = X.cellIndex(me);
            }
            s.diag = s.bx + s.by + s.bz + s.bw;
            bool pinned = rho > 0.0f && pinnedAt(X, X.cellIndex(me));
            s.dx = s.diag + (pinned ? PIN : 0.0f);
            s.dy = wmax(s.diag, 1e-30f);
            s.solving = s.dx > 0.0f;
            s.color = (me.x + me.y) & 1;
            s.t = t;
        }
    for (int sw = 0; sw < 2 * SWEEPS; sw++) {
        for (int li = 0; li < 64; li++) {
            T& s = th[li];
            if (!s.solving || s.color != (sw & 1)) continue;
            int t = s.t;
            float sx = s.bx * pot[t - 1].x + s.by * pot[t + 1].x + s.bz * pot[t - RIM].x + s.bw * pot[t + RIM].x;
            float sy = s.bx * pot[t - 1].y + s.by * pot[t + 1].y + s.bz * pot[t - RIM].y + s.bw * pot[t + RIM].y;
            float nx = mixf(pot[t].x, (sx - s.rhs.x) / s.dx, SMOOTH_OMEGA);
            float ny = mixf(pot[t].y, (sy - s.rhs.y) / s.dy, SMOOTH_OMEGA);
            pot[t] = V2{nx, s.diag > 0.0f ? ny : pot[t].y};
        }
    }
    for (int li = 0; li < 64; li++) {
        T& s = th[li];
        if (!s.solving) continue;
        X.fv(2u * s.idx)[0] = pot[s.t].x;
        X.fv(2u * s.idx + 1u)[0] = pot[s.t].y;
    }
}

void pass_relax(Ctx& X, bool shifted) {
    uint32_t groups = shifted ? X.B + X.L.edge_tiles : X.B;
    for (uint32_t wid = 0; wid < groups; wid++) relaxTile(X, wid, shifted ? BLOCK / 2 : 0);
}

// restrictLevel, smoothAt, solve, prolong, prolongFine (fluid.wgsl:2342-2512)
void pass_restrict(Ctx& X) {
    uint32_t l = X.level;
    if (X.activeCount() == 0u || X.converged()) return;
    I2 s = levelSize(X, l);
    for (int y = 0; y < s.y; y++)
        for (int x = 0; x < s.x; x++) {
            I2 c{x, y};
            uint32_t at = levelSlot(X, l, c);
            int span = 1 << l;
            if (span <= BLOCK) {
                I2 b{c.x * span / BLOCK, c.y * span / BLOCK};
                if (X.inBlocks(b) && (X.blocks[X.stateSlot(X.blockIndex(b))] & ACTIVE) == 0u) {
                    std::memset(X.fv(at), 0, 32);
                    continue;
                }
            }
            float fluid = 0.0f, sum = 0.0f;
            bool air = false;
            V2 r{0, 0};
            for (int j = 0; j < 4; j++) {
                I2 k{2 * c.x + (j & 1), 2 * c.y + (j >> 1)};
                float rho = rhoAt(X, l - 1u, k);
                if (rho == 0.0f) air = true;
                else if (rho > 0.0f) {
                    fluid = fluid + 1.0f;
                    sum = sum + rho;
                    V2 rr = residualAt(X, l - 1u, k);
                    r.x = r.x + rr.x;
                    r.y = r.y + rr.y;
                }
            }
            float rho = air ? 0.0f : (fluid > 0.0f ? sum / fluid : -1.0f);
            float* f = X.fv(at);
            f[0] = 0; f[1] = 0;
            f[2] = rho > 0.0f ? r.x * 0.25f : 0.0f;
            f[3] = rho > 0.0f ? r.y * 0.25f : 0.0f;
            float* g = X.fv(at + 1u);
            g[0] = rho; g[1] = 0; g[2] = 0; g[3] = 0;
        }
}

void pass_smooth(Ctx& X, int color) {
    uint32_t l = X.level;
    if (X.activeCount() == 0u || X.converged()) return;
    I2 s = levelSize(X, l);
    for (int y = 0; y < s.y; y++)
        for (int x = 0; x < s.x; x++) {
            I2 c{x, y};
            if (((c.x + c.y) & 1) != color) continue;
            uint32_t at = levelSlot(X, l, c);
            float rho = X.fv(at + 1u)[0];
            if (rho <= 0.0f) continue;
            V2 sum; float diag;
            stencil(X, l, c, rho, &sum, &diag);
            if (diag <= 0.0f) continue;
            float* e = X.fv(at);
            float h2 = (float)(1u << (2u * l));
            float sx = (sum.x - h2 * e[2]) / diag, sy = (sum.y - h2 * e[3]) / diag;
            e[0] = mixf(e[0], sx, 1.0f);
            e[1] = mixf(e[1], sy, 1.0f);
        }
}

void pass_solve(Ctx& X) {
    if (X.converged()) return;
    uint32_t l = X.level;
    I2 size = levelSize(X, l);
    uint32_t n = wmin((uint32_t)(size.x * size.y), WIG_MG_COARSEST);
    std::vector<V2> pot(n), rhs(n);
    std::vector<float> rho(n);
    for (uint32_t j = 0; j < n; j++) {
        I2 c{(int)(j % (uint32_t)size.x), (int)(j / (uint32_t)size.x)};
        float* f = X.fv(levelSlot(X, l, c));
        pot[j] = V2{f[0], f[1]};
        rhs[j] = V2{f[2], f[3]};
        rho[j] = X.fv(levelSlot(X, l, c) + 1u)[0];
    }
    float h2 = (float)(1u << (2u * l));
    auto crho = [&](I2 c) -> float {
        if (c.x < 0 || c.y < 0 || c.x >= size.x || c.y >= size.y) return -1.0f;
        return rho[(uint32_t)c.y * (uint32_t)size.x + (uint32_t)c.x];
    };
    for (int s = 0; s < 2 * COARSE_SWEEPS; s++) {
        for (uint32_t j = 0; j < n; j++) {
            I2 c{(int)(j % (uint32_t)size.x), (int)(j / (uint32_t)size.x)};
            float r0 = rho[j];
            if (((c.x + c.y) & 1) != (s & 1) || r0 <= 0.0f) continue;
            V2 sum{0, 0};
            float diag = 0.0f;
            for (int d = 0; d < 4; d++) {
                I2 o = Ctx::beside(c, d);
                float r = crho(o);
                if (r < 0.0f) continue;
                float beta = faceBeta(r0, r);
                V2 p = pot[(uint32_t)o.y * (uint32_t)size.x + (uint32_t)o.x];
                sum.x = sum.x + beta * p.x;
                sum.y = sum.y + beta * p.y;
                diag = diag + beta;
            }
            if (diag > 0.0f) {
                pot[j].x = mixf(pot[j].x, (sum.x - h2 * rhs[j].x) / diag, OMEGA);
                pot[j].y = mixf(pot[j].y, (sum.y - h2 * rhs[j].y) / diag, OMEGA);
            }
        }
    }
    for (uint32_t j = 0; j < n; j++) {
        I2 c{(int)(j % (uint32_t)size.x), (int)(j / (uint32_t)size.x)};
        float* f = X.fv(levelSlot(X, l, c));
        f[0] = pot[j].x; f[1] = pot[j].y; f[2] = rhs[j].x; f[3] = rhs[j].y;
    }
}

void pass_prolong(Ctx& X) {
    uint32_t l = X.level;
    if (X.activeCount() == 0u || X.converged()) return;
    I2 s = levelSize(X, l);
    for (int y = 0; y < s.y; y++)
        for (int x = 0; x < s.x; x++) {
            I2 c{x, y};
            uint32_t at = levelSlot(X, l, c);
            if (X.fv(at + 1u)[0] > 0.0f) {
                V2 e = prolonged(X, l, c);
                float* f = X.fv(at);
                f[0] = f[0] + e.x;
                f[1] = f[1] + e.y;
            }
        }
}

void pass_prolongFine(Ctx& X) {
    if (X.converged()) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = 2u * X.cellIndex(c);
        if (X.fv(i)[2] > 0.0f) {
            V2 e = prolonged(X, 0, c);
            X.fv(i)[0] = X.fv(i)[0] + e.x;
            X.fv(i + 1u)[0] = X.fv(i + 1u)[0] + e.y;
        }
    });
}

// The conjugate gradients' block sums (fluid.wgsl:2628-2661): a tree over the
// 64 cells of a block into its slot, then one over 256 threads' strided
// runs of the blocks in index order.
void sumBlock(Ctx& X, I2 b, const float vx[64], const float vy[64]) {
    float wx[64], wy[64];
    for (int i = 0; i < 64; i++) { wx[i] = vx[i]; wy[i] = vy[i]; }
    for (int h = 32; h > 0; h >>= 1)
        for (int li = 0; li < h; li++) { wx[li] = wx[li] + wx[li + h]; wy[li] = wy[li] + wy[li + h]; }
    float* slot = X.cg + 4u * (size_t)(X.C + X.blockIndex(b));
    slot[0] = wx[0]; slot[1] = wy[0]; slot[2] = 0; slot[3] = 0;
}
V2 sumBlocks(Ctx& X) {
    float wx[256], wy[256];
    for (uint32_t li = 0; li < 256; li++) {
        float sx = 0.0f, sy = 0.0f;
        for (uint32_t k = li; k < X.B; k += 256u) {
            if ((X.blocks[X.stateSlot(k)] & ACTIVE) != 0u) {
                sx = sx + X.cg[4u * (size_t)(X.C + k)];
                sy = sy + X.cg[4u * (size_t)(X.C + k) + 1u];
            }
        }
        wx[li] = sx; wy[li] = sy;
    }
    for (int h = 128; h > 0; h >>= 1)
        for (int li = 0; li < h; li++) { wx[li] = wx[li] + wx[li + h]; wy[li] = wy[li] + wy[li + h]; }
    return V2{wx[0], wy[0]};
}
// The FP64 forms (WIG_STEP_F64_DOTS, and the norms of WIG_STEP_TOLERANCE):
// the same two trees in double, the block partials kept per block index.
std::vector<double> g_part64;
double tree64(double* w, int n) {
    for (int h = n / 2; h > 0; h >>= 1)
        for (int li = 0; li < h; li++) w[li] = w[li] + w[li + h];
    return w[0];
}
// Sums of the partials of component `comp` (of 2) over the active blocks in
// index order: 256 strided runs, then a tree.
double sumBlocks64(Ctx& X, int comp) {
    double w[256];
    for (uint32_t li = 0; li < 256; li++) {
        double s = 0.0;
        for (uint32_t k = li; k < X.B; k += 256u)
            if ((X.blocks[X.stateSlot(k)] & ACTIVE) != 0u) s = s + g_part64[2u * k + (uint32_t)comp];
        w[li] = s;
    }
    return tree64(w, 256);
}
void ensure64(Ctx& X) {
    if (g_part64.size() != 2u * X.B) g_part64.assign(2u * X.B, 0.0);
}

void pass_cgRho(Ctx& X) {
    if (X.converged()) return;
    uint32_t na = X.activeCount();
    if (X.f64_dots) ensure64(X);
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        float vx[64], vy[64];
        double dx[64], dy[64];
        for (int li = 0; li < 64; li++) {
            I2 c{b.x * BLOCK + li % BLOCK, b.y * BLOCK + li / BLOCK};
            vx[li] = 0; vy[li] = 0; dx[li] = 0.0; dy[li] = 0.0;
            if (X.inWorld(c) && X.gridAt(c).z > 0.0f) {
                uint32_t i = X.cellIndex(c);
                float z = X.fv(2u * i)[0];
                float* g = X.cg + 4u * (size_t)i;
                vx[li] = g[1] * z;
                vy[li] = g[3] * z;
                dx[li] = (double)g[1] * (double)z;
                dy[li] = (double)g[3] * (double)z;
            }
        }
        sumBlock(X, b, vx, vy);
        if (X.f64_dots) {
            g_part64[2u * X.blockIndex(b)] = tree64(dx, 64);
            g_part64[2u * X.blockIndex(b) + 1u] = tree64(dy, 64);
        }
    }
}
void sums64(Ctx& X, double* sx, double* sy) {
    *sx = sumBlocks64(X, 0);
    *sy = sumBlocks64(X, 1);
}
// The FP64 form's CG scalars, kept beside the f32 sums.
double g_rz = 0.0, g_pq = 0.0, g_alpha = 0.0, g_beta = 0.0;

void pass_cgBeta(Ctx& X) {
    if (X.converged() || X.activeCount() == 0u) return;
    float* at = X.cg + 4u * (size_t)(X.C + X.B);
    if (X.f64_dots) {
        double rz, zq;
        sums64(X, &rz, &zq);
        double beta = (X.cycle == 0u || g_pq <= 0.0) ? 0.0 : -zq / g_pq;
        g_rz = rz;
        g_beta = beta;
        at[0] = (float)rz; at[2] = (float)beta;
        return;
    }
    V2 s = sumBlocks(X);
    V4 was{at[0], at[1], at[2], at[3]};
    float beta = (X.cycle == 0u || was.w <= 0.0f) ? 0.0f : -s.y / was.w;
    at[0] = s.x; at[1] = was.y; at[2] = beta; at[3] = was.w;
}
void pass_cgDirection(Ctx& X) {
    if (X.converged()) return;
    float beta = X.cg[4u * (size_t)(X.C + X.B) + 2u];
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        float* g = X.cg + 4u * (size_t)i;
        float p = 0.0f;
        if (X.fv(2u * i)[2] > 0.0f) {
            if (X.f64_dots) p = (float)((double)X.fv(2u * i)[0] + g_beta * (double)g[2]);
            else p = X.fv(2u * i)[0] + beta * g[2];
        }
        g[2] = p;
    });
}
// applyA (fluid.wgsl:2595-2613)
float applyA(Ctx& X, I2 c, float rho) {
    float sum = 0.0f, diag = 0.0f;
    float share = X.shareAt(c);
    for (int d = 0; d < 4; d++) {
        I2 n = Ctx::beside(c, d);
        float r = rhoAt(X, 0, n);
        if (r < 0.0f) continue;
        float beta = fineBeta(rho, r, share, X.shareAt(n));
        if (r > 0.0f) sum = sum + beta * X.cg[4u * (size_t)X.cellIndex(n) + 2u];
        diag = diag + beta;
    }
    diag = diag + (pinnedAt(X, X.cellIndex(c)) ? PIN : 0.0f);
    return diag * X.cg[4u * (size_t)X.cellIndex(c) + 2u] - sum;
}
void pass_cgApply(Ctx& X) {
    if (X.converged()) return;
    uint32_t na = X.activeCount();
    if (X.f64_dots) ensure64(X);
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        float vx[64], vy[64];
        double dx[64];
        for (int li = 0; li < 64; li++) {
            I2 c{b.x * BLOCK + li % BLOCK, b.y * BLOCK + li / BLOCK};
            vx[li] = 0; vy[li] = 0; dx[li] = 0.0;
            if (!X.inWorld(c)) continue;
            float rho = X.gridAt(c).z;
            uint32_t i = X.cellIndex(c);
            float q = rho > 0.0f ? applyA(X, c, rho) + couplingAt(X, c, PUSH_P0 + X.cycle % 2u) : 0.0f;
            float* g = X.cg + 4u * (size_t)i;
            g[3] = q;
            vx[li] = g[2] * q;
            dx[li] = (double)g[2] * (double)q;
        }
        sumBlock(X, b, vx, vy);
        if (X.f64_dots) {
            g_part64[2u * X.blockIndex(b)] = tree64(dx, 64);
            g_part64[2u * X.blockIndex(b) + 1u] = 0.0;
        }
    }
}
// The bodies' sums of this iteration's direction emptied for the iteration
// after next (fluid.wgsl:2808-2813).
void clearDirectionPushes(Ctx& X) {
    if (!X.pushes) return;
    uint32_t which = PUSH_P0 + X.cycle % 2u;
    for (uint32_t k = 0; k < MAX_BODIES * 6u; k++) X.pushes[pushSlot(k / 6u, which, 0u) + k % 6u] = 0u;
}
void pass_cgAlpha(Ctx& X) {
    if (X.converged() || X.activeCount() == 0u) return;
    float* at = X.cg + 4u * (size_t)(X.C + X.B);
    if (X.f64_dots) {
        double pq, dummy;
        sums64(X, &pq, &dummy);
        g_pq = pq;
        g_alpha = pq <= 0.0 ? 0.0 : g_rz / pq;
        at[1] = (float)g_alpha; at[3] = (float)pq;
        clearDirectionPushes(X);
        return;
    }
    float pq = sumBlocks(X).x;
    V4 was{at[0], at[1], at[2], at[3]};
    at[0] = was.x; at[1] = pq <= 0.0f ? 0.0f : was.x / pq; at[2] = was.z; at[3] = pq;
    clearDirectionPushes(X);
}
void pass_cgUpdate(Ctx& X) {
    X.blocks[X.countSlot(COUNT_RESIDUAL + (X.cycle + 1u) % 3u)] = 0u;
    if (!X.converged()) X.blocks[X.countSlot(COUNT_CYCLES)] += 1u;
    if (X.converged()) return;
    float alpha = X.cg[4u * (size_t)(X.C + X.B) + 1u];
    uint32_t most = 0;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c) || X.gridAt(c).z <= 0.0f) return;
        uint32_t i = X.cellIndex(c);
        float* g = X.cg + 4u * (size_t)i;
        V4 v{g[0], g[1], g[2], g[3]};
        float r, x;
        if (X.f64_dots) {
            r = (float)((double)v.y - g_alpha * (double)v.w);
            x = (float)((double)v.x + g_alpha * (double)v.z);
        } else {
            r = v.y - alpha * v.w;
            x = v.x + alpha * v.z;
        }
        g[0] = x; g[1] = r; g[2] = v.z; g[3] = v.w;
        X.fv(2u * i)[0] = 0.0f;
        X.fv(2u * i)[1] = -r;
        most = wmax(most, bits(std::fabs(r)));
    });
    uint32_t& slot = X.blocks[X.countSlot(COUNT_RESIDUAL + X.cycle % 3u)];
    slot = wmax(slot, most);
    if (X.tol_mode) {
        double rr = norm2Blocks(X, [&](I2 c) -> double {
            uint32_t i = X.cellIndex(c);
            return X.fv(2u * i)[2] > 0.0f ? (double)X.cg[4u * (size_t)i + 1u] : 0.0;
        });
        X.rel = X.bnorm2 > 0.0 ? std::sqrt(rr / X.bnorm2) : 0.0;
    }
}
void pass_cgFinish(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        X.fv(2u * i)[0] = X.cg[4u * (size_t)i];
        X.gw(i, G_REGION) = 0u;
    });
}

// projectFace, project (fluid.wgsl:2897-2942)
void pass_project(Ctx& X) {
    uint32_t& most = X.blocks[X.countSlot(COUNT_MOST_CYCLES)];
    most = wmax(most, X.blocks[X.countSlot(COUNT_CYCLES)]);
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        int fs[4][3];
        X.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            I2 at{fs[j][0], fs[j][1]};
            bool isU = fs[j][2] == 1;
            float* face = X.fv(X.faceSlot(X.faceIndex(at, isU)));
            I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
            V4 ga = X.gridAt(a), gb = X.gridAt(at);
            float beta = fineBeta(ga.z, gb.z, X.shareAt(a), X.shareAt(at));
            uint32_t ra = rigidAt(X, a), rb = rigidAt(X, at);
            if (beta > 0.0f) {
                face[0] = face[0] - beta * (gb.x - ga.x);
                face[2] = PROJECTED;
                bool rigid = ra != NONE || rb != NONE;
                face[3] = rigid ? 0.0f : clampf(-beta * (X.driftAt(at) - X.driftAt(a)), -MAX_DRIFT, MAX_DRIFT);
            }
            // a face between the liquid and a free body moves with the body's push (PUSH_F)
            if ((ra == NONE) != (rb == NONE) && (ra != NONE ? gb.z : ga.z) > 0.0f) {
                uint32_t bb = ra != NONE ? ra : rb;
                V3 ch = pushChange(X, bb, PUSH_F);
                V2 m = faceMiddle(at, isU);
                V2 pos = bodyV(X, bb, WIG_BW_POS);
                V2 r{m.x - pos.x, m.y - pos.y};
                face[0] = face[0] + (isU ? ch.x - ch.z * r.y : ch.y + ch.z * r.x);
                face[2] = PROJECTED;
            }
        }
    });
}

// ---------------------------------------------------------------- the bodies' passes

// bodyStart (fluid.wgsl:3079-3084)
void pass_bodyStart(Ctx& X) {
    if (!X.pushes) return;
    for (uint32_t k = 0; k < MAX_BODIES * WIG_BODY_PUSH_WORDS; k++) X.pushes[k] = 0u;
}
// seepLoads, bodyLoads (fluid.wgsl:3094-3139)
void seepLoads(Ctx& X, I2 c, uint32_t b) {
    for (int d = 0; d < 4; d++) {
        I2 q = Ctx::beside(c, d);
        if (!X.inWorld(q) || rigidAt(X, q) == b || X.gridAt(q).z >= 0.0f) continue;
        I2 n{q.x - c.x, q.y - c.y};
        V2 x{((float)c.x + 0.5f) + 0.5f * (float)n.x, ((float)c.y + 0.5f) + 0.5f * (float)n.y};
        addPush(X, b, PUSH_SURFACE, scale3(bodyFaceJ(X, q, c, b), seepAt(X, c, n, b, false, x)));
    }
}
void pass_bodyLoads(Ctx& X) {
    if (!X.motion) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t own = rigidAt(X, c);
        if (own != NONE) { seepLoads(X, c, own); return; }
        V4 g = X.gridAt(c);
        if (g.z <= 0.0f) return;
        V2 mid{(float)c.x + 0.5f, (float)c.y + 0.5f};
        for (int d = 0; d < 4; d++) {
            I2 q = Ctx::beside(c, d);
            uint32_t b = rigidAt(X, q);
            if (b == NONE) continue;
            I2 n{q.x - c.x, q.y - c.y};
            float reach = 1.0f - bodyReach(X, b, I2{-n.x, -n.y});
            V2 surface{mid.x + (float)n.x * reach, mid.y + (float)n.y * reach};
            addPush(X, b, PUSH_SURFACE,
                    scale3(scale3(bodyFaceJ(X, c, q, b), g.z), potentialAt(X, mid) - potentialAt(X, surface)));
        }
    });
}
// bodyDrag (fluid.wgsl:3149-3176)
void pass_bodyDrag(Ctx& X) {
    if (!X.motion) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        uint32_t b = rigidAt(X, c);
        if (!X.inWorld(c) || b == NONE) return;
        V2 pos = bodyV(X, b, WIG_BW_POS);
        float rho = bodyDensity(X, b);
        V3 push{0.0f, 0.0f, 0.0f};
        for (int k = 0; k < 4; k++) {
            bool isU = k < 2;
            int sg = (k & 1) == 1 ? 1 : -1;
            I2 n = isU ? I2{sg, 0} : I2{0, sg};
            if (X.gridAt(I2{c.x + n.x, c.y + n.y}).z <= 0.0f) continue;
            I2 at = isU ? I2{c.x + (k & 1), c.y} : I2{c.x, c.y + (k & 1)};
            V2 x = faceMiddle(at, isU);
            V2 mv = bodyMoving(X, b, x, false);
            float du = (bodyReach(X, b, n) * rho) * (X.fv(X.faceSlot(X.faceIndex(at, isU)))[0] - (isU ? mv.x : mv.y));
            V2 r{x.x - pos.x, x.y - pos.y};
            if (isU) push.x = push.x + du; else push.y = push.y + du;
            push.z = push.z + (isU ? -r.y * du : r.x * du);
        }
        if (push.x != 0.0f || push.y != 0.0f || push.z != 0.0f) addPush(X, b, PUSH_DRAG, push);
    });
}
// bodyFaces (fluid.wgsl:3180-3200)
void pass_bodyFaces(Ctx& X) {
    if (!X.motion) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        int fs[4][3];
        X.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            I2 at{fs[j][0], fs[j][1]};
            bool isU = fs[j][2] == 1;
            I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
            uint32_t ra = rigidAt(X, a), rb = rigidAt(X, at);
            if (ra != NONE || rb != NONE) setBodyFace(X, X.faceIndex(at, isU), at, isU, X.gridAt(a), X.gridAt(at), ra, rb, true);
        }
    });
}
// cgBodyX, cgBodyP, cgBodyF (fluid.wgsl:2819-2845)
void pass_cgBodyX(Ctx& X) {
    if (!X.motion) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (X.inWorld(c) && X.gridAt(c).z > 0.0f) addPressurePush(X, c, X.cg[4u * (size_t)X.cellIndex(c)], PUSH_X);
    });
}
void pass_cgBodyP(Ctx& X) {
    if (!X.motion || X.converged()) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (X.inWorld(c) && X.gridAt(c).z > 0.0f)
            addPressurePush(X, c, X.cg[4u * (size_t)X.cellIndex(c) + 2u], PUSH_P0 + X.cycle % 2u);
    });
}
void pass_cgBodyF(Ctx& X) {
    if (!X.motion) return;
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (X.inWorld(c) && X.gridAt(c).z > 0.0f) addPressurePush(X, c, X.fv(2u * X.cellIndex(c))[0], PUSH_F);
    });
}
// rigidify (fluid.wgsl:3033-3076): each block's cells of its lowest held
// body summed once, the others' added straight into their bodies' words.
void pass_rigidify(Ctx& X) {
    if (!X.motion) return;
    uint32_t na = X.activeCount();
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        uint32_t first = NONE;
        for (int li = 0; li < 64; li++) {
            uint32_t h = heldAt(X, I2{b.x * BLOCK + li % BLOCK, b.y * BLOCK + li / BLOCK});
            if (h != NONE) first = wmin(first, h);
        }
        uint32_t sums[3] = {0u, 0u, 0u};
        for (int li = 0; li < 64; li++) {
            I2 c{b.x * BLOCK + li % BLOCK, b.y * BLOCK + li / BLOCK};
            uint32_t h = heldAt(X, c);
            if (h == NONE) continue;
            int32_t d[3];
            heldPush(X, c, h, d);
            if ((X.blocks[X.stateSlot(X.blockIndex(b))] & NEAR_LIQUID) != 0u) X.motion[liquidSlot(h, 3u)] |= WIG_LIQUID_WET;
            for (int k = 0; k < 3; k++) {
                if (h == first) sums[k] += (uint32_t)d[k];
                else X.motion[liquidSlot(h, (uint32_t)k)] += (uint32_t)d[k];
            }
        }
        if (first != NONE)
            for (uint32_t k = 0; k < 3; k++) X.motion[liquidSlot(first, k)] += sums[k];
    }
}
// bodyPush (fluid.wgsl:3205-3218)
void pass_bodyPush(Ctx& X) {
    if (!X.motion) return;
    for (uint32_t b = 0; b < MAX_BODIES; b++) {
        V3 ch = add3(add3(pushChangeFree(X, b, PUSH_SURFACE), pushChangeFree(X, b, PUSH_DRAG)), pushChangeFree(X, b, PUSH_F));
        if (ch.x == 0.0f && ch.y == 0.0f && ch.z == 0.0f) continue;
        X.motion[liquidSlot(b, 0u)] += (uint32_t)f2i(rnd_even(ch.x * RIGID_FIX));
        X.motion[liquidSlot(b, 1u)] += (uint32_t)f2i(rnd_even(ch.y * RIGID_FIX));
        X.motion[liquidSlot(b, 2u)] += (uint32_t)f2i(rnd_even(ch.z * RIGID_FIX));
    }
}

// extrapolateFace (fluid.wgsl:3226-3265)
void pass_extrapolate(Ctx& X, uint32_t layer) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        int fs[4][3];
        X.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            I2 at{fs[j][0], fs[j][1]};
            bool isU = fs[j][2] == 1;
            float* face = X.fv(X.faceSlot(X.faceIndex(at, isU)));
            I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
            if (face[2] != 1.0f || X.gridAt(a).z != 0.0f || X.gridAt(at).z != 0.0f) continue;
            float reached = layer == 2u ? 1.5f : PROJECTED;
            float sum = 0.0f, n = 0.0f;
            for (int d = 0; d < 4; d++) {
                I2 q = Ctx::beside(at, d);
                if (!X.faceInWorld(q, isU)) continue;
                float* g = X.fv(X.faceSlot(X.faceIndex(q, isU)));
                if (g[2] >= reached) { sum = sum + g[0]; n = n + 1.0f; }
            }
            if (n > 0.0f) {
                face[0] = sum / n;
                face[2] = layer == 2u ? 1.25f : 1.5f;
            }
        }
    });
}

// advect (fluid.wgsl:3470-3694)
struct Sample { float now, before, weight, drift; V2 gradient; };
Sample sampleAxis(Ctx& X, V2 s, bool isU) {
    float fx0 = std::floor(s.x), fy0 = std::floor(s.y);
    I2 b{f2i(fx0), f2i(fy0)};
    V2 f{s.x - fx0, s.y - fy0};
    float ax = 0.0f, ay = 0.0f;
    Sample r{0, 0, 0, 0, {0, 0}};
    int held = 0;
    V2 g{0, 0};
    for (int j = 0; j < 4; j++) {
        int ox = j & 1, oy = j >> 1;
        float w = (ox == 1 ? f.x : 1.0f - f.x) * (oy == 1 ? f.y : 1.0f - f.y);
        V2 dw{(ox == 1 ? 1.0f : -1.0f) * (oy == 1 ? f.y : 1.0f - f.y), (ox == 1 ? f.x : 1.0f - f.x) * (oy == 1 ? 1.0f : -1.0f)};
        I2 at{b.x + ox, b.y + oy};
        if (!X.faceInWorld(at, isU)) continue;
        float* face = X.fv(X.faceSlot(X.faceIndex(at, isU)));
        r.drift = r.drift + w * face[3];
        if (face[2] > 0.0f) {
            ax = ax + w * face[0];
            ay = ay + w * face[1];
            r.weight = r.weight + w;
            g.x = g.x + dw.x * face[0];
            g.y = g.y + dw.y * face[0];
            held += face[2] == PROJECTED ? 1 : 0;
        }
    }
    if (r.weight > 0.0f) {
        r.now = ax / r.weight;
        r.before = ay / r.weight;
    }
    r.gradient = held == 4 ? g : V2{0, 0};
    return r;
}
bool isObstacle(Ctx& X, V2 pos) {
    I2 c{f2i(std::floor(pos.x)), f2i(std::floor(pos.y))};
    if (X.gridAt(c).z < 0.0f) return true;
    uint32_t k = X.kindOfCell(X.cellIndex(c));
    return k == WIG_KIND_SOLID || k == WIG_KIND_POWDER;
}
// shutAt, escapesTo (fluid.wgsl:1468-1470, :3535-3541)
bool escapesTo(Ctx& X, I2 q, uint32_t side) {
    if (!X.inWorld(q) || X.gridAt(q).z < 0.0f || rigidAt(X, q) != NONE) return false;
    uint32_t cup = cupOf(X, X.cellIndex(q));
    return cup == NONE || cup == side;
}
V2 escape(Ctx& X, V2 pos) {
    if (!isObstacle(X, pos)) return pos;
    I2 c{f2i(std::floor(pos.x)), f2i(std::floor(pos.y))};
    const uint32_t side = X.inWorld(c) ? cupBefore(X, X.cellIndex(c)) : NONE;
    V2 best = pos;
    float bestD = 1e9f;
    for (int n = 0; n < 8; n++) {
        int m = n + (n >= 4 ? 1 : 0);
        I2 at{c.x + m % 3 - 1, c.y + m / 3 - 1};
        if (!escapesTo(X, at, side)) continue;
        V2 inside{clampf(pos.x, (float)at.x + 0.02f, (float)at.x + 0.98f), clampf(pos.y, (float)at.y + 0.02f, (float)at.y + 0.98f)};
        float dx = pos.x - inside.x, dy = pos.y - inside.y;
        float d = std::sqrt(dx * dx + dy * dy);
        if (d < bestD) { bestD = d; best = inside; }
    }
    if (bestD < 1e9f) return best;
    const I2 ways[4] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}};
    I2 way = ways[0];
    int nearest = ESCAPE_REACH + 1;
    for (int n = 0; n < 4; n++) {
        I2 dir = ways[n];
        for (int r = 2; r < nearest; r++) {
            I2 q{c.x + dir.x * r, c.y + dir.y * r};
            if (!isObstacle(X, V2{(float)q.x + 0.5f, (float)q.y + 0.5f}) && escapesTo(X, q, side)) {
                nearest = r;
                way = dir;
                break;
            }
        }
    }
    return X.inWorld(I2{c.x + way.x, c.y + way.y}) ? V2{pos.x + (float)way.x, pos.y + (float)way.y} : pos;
}
V2 clampSpeed(V2 v) {
    float s = std::sqrt(v.x * v.x + v.y * v.y);
    if (s > LIQUID_MAX_SPEED) {
        float k = LIQUID_MAX_SPEED / s;
        return V2{v.x * k, v.y * k};
    }
    return v;
}
V2 slipOf(Ctx& X, const Particle& q) {
    uint32_t i = X.cellIndex(X.cellOf(q.pos));
    uint32_t n = X.gw(i, G_COUNT);
    if (n < 2u) return V2{0, 0};
    float mean = (float)X.gw(i, G_MASS) / (FIX * (float)n);
    float lighter = (mean - X.liquidDensity(q.word, q.temp)) / wmax(mean, 1e-3f);
    V2 pull = X.pullAt(q.pos);
    float wgt = X.elem(WATER).weight;
    return V2{-pull.x / wgt * SLIP * lighter, -pull.y / wgt * SLIP * lighter};
}
void pass_advect(Ctx& X) {
    uint32_t live = X.partsLive();
    for (uint32_t k = 0; k < live; k++) {
        Particle q = X.toParticle(X.parts, k);
        const wig_elem& e = X.elem(wordType(q.word));
        V2 orig = q.pos;
        q.pos = escape(X, q.pos);
        Sample u = sampleAxis(X, V2{q.pos.x - 0.0f, q.pos.y - 0.5f}, true);
        Sample v = sampleAxis(X, V2{q.pos.x - 0.5f, q.pos.y - 0.0f}, false);
        V2 flow{u.weight > 0.0f ? u.now : q.vel.x, v.weight > 0.0f ? v.now : q.vel.y};
        V2 vel = clampSpeed(flow);
        V4 affine{AFFINE_KEEP * u.gradient.x, AFFINE_KEEP * u.gradient.y, AFFINE_KEEP * v.gradient.x, AFFINE_KEEP * v.gradient.y};
        V2 cs = clampSpeed(vel);
        V2 sl = slipOf(X, q);
        V2 travel{cs.x + clampf(u.drift + sl.x, -MAX_DRIFT, MAX_DRIFT), cs.y + clampf(v.drift + sl.y, -MAX_DRIFT, MAX_DRIFT)};
        int steps = wmin(wmax(f2i(std::ceil(wmax(std::fabs(travel.x), std::fabs(travel.y)) * 2.0f)), 1), ADVECT_STEPS);
        V2 d{travel.x / (float)steps, travel.y / (float)steps};
        V2 pos = q.pos;
        float impact = 0.0f;
        for (int s = 0; s < steps; s++) {
            V2 nx{pos.x + d.x, pos.y + 0.0f};
            if (d.x != 0.0f && isObstacle(X, nx)) {
                if (vel.x * d.x > 0.0f) { impact = wmax(impact, std::fabs(vel.x)); vel.x = 0.0f; }
                d.x = 0.0f;
            } else pos = nx;
            V2 ny{pos.x + 0.0f, pos.y + d.y};
            if (d.y != 0.0f && isObstacle(X, ny)) {
                if (vel.y * d.y > 0.0f) { impact = wmax(impact, std::fabs(vel.y)); vel.y = 0.0f; }
                d.y = 0.0f;
            } else pos = ny;
        }
        if (!X.isActiveBlock(Ctx::divI(X.cellOf(pos), BLOCK))) {
            pos = q.pos;
            if (!X.isActiveBlock(Ctx::divI(X.cellOf(pos), BLOCK))) pos = orig;
        }
        uint32_t* m = X.item(X.parts, k);
        m[0] = bits(pos.x); m[1] = bits(pos.y); m[2] = bits(vel.x); m[3] = bits(vel.y);
        uint32_t* a = X.item(X.parts, 2u * X.cap + k);
        a[0] = bits(affine.x); a[1] = bits(affine.y); a[2] = bits(affine.z); a[3] = bits(affine.w);
        float* left = X.fv(2u * X.cellIndex(X.cellOf(q.pos)));
        if (left[2] > 0.0f) {
            V2 pull = X.pullAt(q.pos);
            bool falling = left[0] < 0.5f * left[2] * std::sqrt(pull.x * pull.x + pull.y * pull.y);
            X.gw(X.cellIndex(X.cellOf(pos)), G_CAME) |= falling ? CAME_FALLING : CAME_PRESSING;
        }
        if ((e.flags & F_IMPACT) != 0u && impact > IMPACT_SPEED) X.item(X.parts, X.cap + k)[0] = wordWith(q.word, FL_BURN);
    }
}

// sortCount, scanBlocks, scanTotals, scanFinish, scatter (fluid.wgsl:3700-3808)
void pass_sortCount(Ctx& X) {
    uint32_t live = X.partsLive();
    for (uint32_t k = 0; k < live; k++) {
        uint32_t* m = X.item(X.parts, k);
        uint32_t i = X.cellIndex(X.cellOf(V2{flt(m[0]), flt(m[1])}));
        X.item(X.parts, X.cap + k)[3] = X.gw(i, G_SORT)++;
    }
}
void pass_scanBlocks(Ctx& X) {
    uint32_t na = X.activeCount();
    uint32_t fall0 = 4u << (X.P->frame & 1u);
    for (uint32_t wid = 0; wid < na; wid++) {
        I2 b = X.activeBlock(wid);
        uint32_t run = 0;
        for (int li = 0; li < 64; li++) {
            I2 c{b.x * BLOCK + li % BLOCK, b.y * BLOCK + li / BLOCK};
            if (!X.inWorld(c)) continue;
            uint32_t i = X.cellIndex(c);
            uint32_t n = X.gw(i, G_SORT);
            X.gw(i, G_START) = run;
            run += n;
            uint32_t came = X.gw(i, G_CAME);
            X.gw(i, G_CAME) = 0u;
            if (came == CAME_FALLING) {
                float* w = X.fv(2u * i + 1u) + 3;
                *w = (float)(f2u(*w) | fall0);
            }
        }
        X.blocks[X.totalSlot(wid)] = run;
    }
}
void pass_scanTotals(Ctx& X) {
    uint32_t na = X.activeCount();
    uint32_t run = 0;
    for (uint32_t j = 0; j < na; j++) {
        uint32_t t = X.blocks[X.totalSlot(j)];
        X.blocks[X.totalSlot(j)] = run;
        run += t;
    }
    X.sorted[0] = run;
    X.blocks[X.countSlot(COUNT_PARTICLES)] = run;
}
void pass_scanFinish(Ctx& X) {
    forActiveCells(X, [&](uint32_t wid, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        X.gw(X.cellIndex(c), G_START) += X.blocks[X.totalSlot(wid)];
    });
}
void pass_scatter(Ctx& X) {
    uint32_t live = X.partsLive();
    for (uint32_t k = 0; k < live; k++) {
        uint32_t* m = X.item(X.parts, k);
        uint32_t* s = X.item(X.parts, X.cap + k);
        uint32_t i = X.cellIndex(X.cellOf(V2{flt(m[0]), flt(m[1])}));
        uint32_t at = X.gw(i, G_START) + s[3];
        if (at < X.cap) {
            std::memcpy(X.item(X.sorted, at), m, 16);
            std::memcpy(X.item(X.sorted, X.cap + at), s, 16);
            std::memcpy(X.item(X.sorted, 2u * X.cap + at), X.item(X.parts, 2u * X.cap + k), 16);
        }
    }
}

// rasterClaims, raster, unpaint (fluid.wgsl:3880-4182), no people, no air source.
bool vacated(Ctx& X, uint32_t j) { return X.kindOfCell(j) == WIG_KIND_LIQUID && X.gw(j, G_SORT) == 0u; }
uint32_t airTo(Ctx& X, I2 c, bool gas) {
    if (!gas && X.gridAt(c).z > 0.0f) return NONE;
    static const I2 airOrder[8] = {{0, -1}, {-1, 0}, {1, 0}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
    static const I2 gasOrder[8] = {{0, -1}, {-1, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {1, 1}, {0, 1}};
    for (int n = 0; n < 8; n++) {
        I2 o = gas ? gasOrder[n] : airOrder[n];
        I2 at{c.x + o.x, c.y + o.y};
        if (!X.inWorld(at)) continue;
        uint32_t j = X.cellIndex(at);
        if (vacated(X, j) || (gas && X.cellType(j) == AIR && X.gw(j, G_SORT) == 0u)) return j;
    }
    return NONE;
}
void pass_rasterClaims(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        uint32_t to = NONE;
        uint32_t t = X.cellType(i);
        if (X.gw(i, G_SORT) > 0u) {
            if (t == AIR) to = airTo(X, c, false);
            else if (X.elem(t).kind == WIG_KIND_GAS && X.gridAt(c).z >= 0.0f) to = airTo(X, c, true);
        }
        X.gw(i, G_AIR_TO) = to;
        if (to != NONE) {
            uint32_t& w = X.gw(to, G_TAKEN);
            w = wmax(w, takenBy(i));
        }
    });
}
inline uint64_t exact_add(uint64_t w, float x) {
    // exactParts(x, EXACT_FINE) (common.wgsl:1383-1393) added into a 64-bit two's complement sum.
    float s = rnd_even(clampf(x * EXACT_FINE, -9.2e18f, 9.2e18f));
    uint32_t lo, hi;
    if (std::fabs(s) < 2147483648.0f) {
        int32_t v = (int32_t)s;
        lo = (uint32_t)v;
        hi = v < 0 ? 0xffffffffu : 0u;
    } else {
        float h = std::floor(s / 4294967296.0f);
        lo = f2u(s - h * 4294967296.0f);
        hi = (uint32_t)f2i(h);
    }
    uint32_t wl = (uint32_t)w, wh = (uint32_t)(w >> 32);
    uint32_t nl = wl + lo;
    uint32_t nh = wh + hi + (nl < lo ? 1u : 0u);
    return ((uint64_t)nh << 32) | nl;
}
inline float exact_value(uint64_t w, float scale) {
    int32_t l = (int32_t)(uint32_t)w, h = (int32_t)(uint32_t)(w >> 32);
    if ((h == 0 && l >= 0) || (h == -1 && l < 0)) return (float)l / scale;
    return ((float)h * 4294967296.0f + (float)(uint32_t)w) / scale;
}
void pass_raster(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        uint32_t n = X.gw(i, G_SORT);
        if (n == 0u) return;
        uint32_t start = X.gw(i, G_START);
        uint32_t* vp = X.cellv(i);
        uint32_t v[4] = {vp[0], vp[1], vp[2], vp[3]};
        uint32_t t = wordType(v[0]);
        bool drawn = false;
        if (X.elem(t).kind == WIG_KIND_LIQUID) {
            drawn = true;
        } else if (t == AIR || (X.elem(t).kind == WIG_KIND_GAS && X.gridAt(c).z >= 0.0f)) {
            uint32_t to = X.gw(i, G_AIR_TO);
            if (to != NONE && to < X.C && X.gw(to, G_TAKEN) == takenBy(i)) {
                if (X.cellType(to) == AIR) {  // pushGasOut: into the (unbound) air source
                    uint32_t* gp = X.gasPairPtr(to);
                    gp[0] = 0u; gp[1] = 0u;
                }
                std::memcpy(X.cellv(to), v, 16);
                uint32_t* gi = X.gasPairPtr(i);
                uint32_t* gt = X.gasPairPtr(to);
                gt[0] = gi[0]; gt[1] = gi[1];
                gi[0] = 0u; gi[1] = 0u;
                drawn = true;
            } else if (t == AIR) {
                uint32_t* gp = X.gasPairPtr(i);
                gp[0] = 0u; gp[1] = 0u;
                drawn = true;
            }
        }
        if (!drawn) {
            X.gw(i, G_DEST) = DEST_KEEP;
            return;
        }
        uint32_t kinds[RASTER_KINDS] = {NONE, NONE, NONE, NONE};
        uint32_t counts[RASTER_KINDS] = {0, 0, 0, 0};
        for (uint32_t k = start; k < start + n && k < X.cap; k++) {
            uint32_t pt = wordType(X.item(X.sorted, X.cap + k)[0]);
            uint32_t at = RASTER_KINDS;
            for (uint32_t m = 0; m < RASTER_KINDS; m++)
                if (kinds[m] == pt) at = m;
            if (at == RASTER_KINDS && pt < kinds[RASTER_KINDS - 1u]) {
                at = RASTER_KINDS - 1u;
                kinds[at] = pt;
                counts[at] = 0u;
                while (at > 0u && kinds[at - 1u] > kinds[at]) {
                    std::swap(kinds[at - 1u], kinds[at]);
                    std::swap(counts[at - 1u], counts[at]);
                    at--;
                }
            }
            if (at < RASTER_KINDS) counts[at]++;
        }
        uint32_t most = kinds[0], votes = counts[0];
        for (uint32_t m = 1; m < RASTER_KINDS; m++)
            if (counts[m] > votes) { most = kinds[m]; votes = counts[m]; }
        uint32_t word = 0, lowest = NONE, solute = 0, soluteId = NONE;
        bool solutes = holdsSolute(most);
        for (uint32_t k = start; k < start + n && k < X.cap; k++) {
            uint32_t* st = X.item(X.sorted, X.cap + k);
            if (wordType(st[0]) == most && (lowest == NONE || st[2] < lowest)) { word = st[0]; lowest = st[2]; }
            if (solutes && wordType(st[0]) == most && wordAux(st[0]) != 0u && (soluteId == NONE || st[2] < soluteId)) {
                solute = wordAux(st[0]);
                soluteId = st[2];
            }
        }
        if (solutes) word = packWord(wordType(word), solute, wordLife(word), wordShade(word), wordFlags(word));
        float lx = 0.0f, ly = 0.0f;
        uint64_t heat = 0, capa = 0, vx = 0, vy = 0;
        for (uint32_t k = start; k < start + n && k < X.cap; k++) {
            uint32_t* st = X.item(X.sorted, X.cap + k);
            uint32_t pt = wordType(st[0]);
            if (pt == most && wordAux(st[0]) == wordAux(word)) {
                lx = lx + (float)wordLife(st[0]);
                ly = ly + 1.0f;
            } else if (pt == most && solutes && wordAux(st[0]) == 0u) {
                ly = ly + 1.0f;
            }
            float hc = wmax(X.elem(pt).heat_cap, 1e-6f);
            heat = exact_add(heat, hc * flt(st[1]));
            capa = exact_add(capa, hc);
            uint32_t* mo = X.item(X.sorted, k);
            vx = exact_add(vx, flt(mo[2]));
            vy = exact_add(vy, flt(mo[3]));
        }
        X.seedRng(i, X.P->frame, X.P->seed ^ 0x7a57u);
        uint32_t life = wmin(f2u(std::floor(lx / ly + X.rnd())), 255u);
        word = packWord(wordType(word), wordAux(word), life, wordShade(word), wordFlags(word));
        float temp = exact_value(heat, EXACT_FINE) / exact_value(capa, EXACT_FINE);
        float velx = exact_value(vx, EXACT_FINE) / (float)n, vely = exact_value(vy, EXACT_FINE) / (float)n;
        vp[0] = wordWith(word, FL_DRAWN);
        vp[1] = bits(temp);
        vp[2] = pack2x16(velx, vely);
        vp[3] = liquidW(i, n);
        X.gw(i, G_TYPE) = drawnAs(word) | (life << 16u);
    });
}
void pass_unpaint(Ctx& X) {
    forActiveCells(X, [&](uint32_t, I2 c, uint32_t) {
        if (!X.inWorld(c)) return;
        uint32_t i = X.cellIndex(c);
        uint32_t* v = X.cellv(i);
        if (X.kindOfCell(i) == WIG_KIND_LIQUID && X.gw(i, G_SORT) == 0u && X.gw(i, G_TAKEN) == 0u) {
            float t = X.wordTempOf(v);
            v[0] = AIR; v[1] = bits(t); v[2] = 0u; v[3] = 0u;
            uint32_t* gp = X.gasPairPtr(i);
            gp[0] = 0u; gp[1] = 0u;
        }
    });
}

// ---------------------------------------------------------------- layout

int layout(const wig_world_desc* d, wig_world_layout* L) {
    if (!d || !L || d->width == 0 || d->height == 0 || d->width > 65536 || d->height > 65536) return WIG_E_ARG;
    std::memset(L, 0, sizeof(*L));
    uint64_t W = d->width, H = d->height, C = W * H;
    if (C > (1ull << 30)) return WIG_E_ARG;
    uint64_t F = (W + 1) * H + W * (H + 1);
    L->width = (uint32_t)W; L->height = (uint32_t)H;
    L->liquid_per_cell = d->liquid_per_cell ? d->liquid_per_cell : 4u;
    L->capacity = d->capacity ? d->capacity : (uint32_t)std::ceil((double)C * L->liquid_per_cell * 1.25);
    L->cell_count = (uint32_t)C; L->face_count = (uint32_t)F;
    L->blocks_wide = (uint32_t)((W + 7) / 8);
    L->block_count = L->blocks_wide * (uint32_t)((H + 7) / 8);
    L->edge_tiles = (uint32_t)((W + 7) / 8 + (H + 7) / 8 + 1);
    uint64_t levelCells = 0;
    for (uint32_t l = 1; l <= WIG_MG_LEVELS; l++) {
        uint64_t lw = (W + (1ull << l) - 1) >> l, lh = (H + (1ull << l) - 1) >> l;
        L->level_w[l - 1] = (uint32_t)lw; L->level_h[l - 1] = (uint32_t)lh;
        L->levels = l;
        levelCells += lw * lh;
        if (lw * lh <= WIG_MG_COARSEST) break;
    }
    L->cells_bytes = 16ull * (C + (C + 1) / 2);
    L->particles_bytes = 16ull + 48ull * L->capacity;
    L->counters_bytes = 4ull * (11ull * C + 2ull * F);
    L->field_bytes = 16ull * ((C + levelCells) * 2ull + F + 2ull * ((F + 3) / 4));
    L->blocks_bytes = 4ull * (5ull * L->block_count + WIG_FLUID_STATS);
    L->cg_bytes = 16ull * (C + L->block_count + 1);
    return WIG_OK;
}

// The bodies' buffers bound by wo_bind_bodies (null: none).
uint32_t* g_motion = nullptr;
uint32_t* g_pushes = nullptr;
uint32_t* g_stamps = nullptr;

void setup(Ctx& X, const wig_world_layout& L, const wig_params* P, const wig_elem* E, uint32_t nE, wig_fluid_buffers* b) {
    X.L = L; X.P = P; X.E = E; X.nE = nE;
    X.motion = g_motion;
    X.pushes = g_pushes;
    X.stamps = g_stamps;
    X.cells = (uint32_t*)b->cells; X.sorted = (uint32_t*)b->sorted; X.parts = (uint32_t*)b->parts;
    X.counters = (uint32_t*)b->counters; X.field = (float*)b->field; X.blocks = (uint32_t*)b->blocks; X.cg = (float*)b->cg;
    X.W = (int)L.width; X.H = (int)L.height;
    X.C = L.cell_count; X.F = L.face_count; X.B = L.block_count; X.BW = L.blocks_wide;
    X.cap = L.capacity; X.ppc = L.liquid_per_cell;
    uint32_t at = 2u * X.C + X.F + 2u * ((X.F + 3u) / 4u);
    X.levelStartV[0] = 0;
    for (uint32_t l = 1; l <= WIG_MG_LEVELS; l++) {
        X.levelStartV[l] = at;
        if (l <= L.levels) at += 2u * L.level_w[l - 1] * L.level_h[l - 1];
    }
}

void run_pass(Ctx& X, int pass) {
    switch (pass) {
    case WIG_PASS_SYNC: pass_sync(X, true); break;
    case WIG_PASS_SYNC_MARKS: pass_sync(X, false); break;
    case WIG_PASS_SYNC_PARTICLES: pass_syncParticles(X); break;
    case WIG_PASS_SYNC_SEED: pass_syncSeed(X); break;
    case WIG_PASS_COMPACT: pass_compact(X); break;
    case WIG_PASS_RETIRE: pass_retire(X); break;
    case WIG_PASS_CLEAR: pass_clear(X); break;
    case WIG_PASS_GATHER: pass_gather(X); break;
    case WIG_PASS_SEAL_JOIN: pass_sealJoin(X); break;
    case WIG_PASS_SEAL_ANCHOR: pass_sealAnchor(X); break;
    case WIG_PASS_CLASSIFY: pass_classify(X); break;
    case WIG_PASS_SET_FACES: pass_setFaces(X); break;
    case WIG_PASS_VISCOSITY_RED: pass_viscosity(X, 0); break;
    case WIG_PASS_VISCOSITY_BLACK: pass_viscosity(X, 1); break;
    case WIG_PASS_UNPRESS: pass_viscosity(X, 2); break;
    case WIG_PASS_DIVERGENCE: pass_divergence(X); break;
    case WIG_PASS_CG_START: pass_cgStart(X); break;
    case WIG_PASS_CG_JOIN: pass_cgJoin(X); break;
    case WIG_PASS_CG_ANCHOR: pass_cgAnchor(X); break;
    case WIG_PASS_CG_RESIDUAL: pass_cgResidual(X); break;
    case WIG_PASS_CG_PREPARE: pass_cgPrepare(X); break;
    case WIG_PASS_RELAX_RIMS: pass_relaxRims(X); break;
    case WIG_PASS_RELAX: pass_relax(X, false); break;
    case WIG_PASS_RELAX_SHIFTED: pass_relax(X, true); break;
    case WIG_PASS_RESTRICT: pass_restrict(X); break;
    case WIG_PASS_SMOOTH_RED: pass_smooth(X, 0); break;
    case WIG_PASS_SMOOTH_BLACK: pass_smooth(X, 1); break;
    case WIG_PASS_SOLVE: pass_solve(X); break;
    case WIG_PASS_PROLONG: pass_prolong(X); break;
    case WIG_PASS_PROLONG_FINE: pass_prolongFine(X); break;
    case WIG_PASS_CG_RHO: pass_cgRho(X); break;
    case WIG_PASS_CG_BETA: pass_cgBeta(X); break;
    case WIG_PASS_CG_DIRECTION: pass_cgDirection(X); break;
    case WIG_PASS_CG_APPLY: pass_cgApply(X); break;
    case WIG_PASS_CG_ALPHA: pass_cgAlpha(X); break;
    case WIG_PASS_CG_UPDATE: pass_cgUpdate(X); break;
    case WIG_PASS_CG_FINISH: pass_cgFinish(X); break;
    case WIG_PASS_PROJECT: pass_project(X); break;
    case WIG_PASS_EXTRAPOLATE: pass_extrapolate(X, 1u); break;
    case WIG_PASS_EXTRAPOLATE_FURTHER: pass_extrapolate(X, 2u); break;
    case WIG_PASS_ADVECT: pass_advect(X); break;
    case WIG_PASS_SORT_COUNT: pass_sortCount(X); break;
    case WIG_PASS_SCAN_BLOCKS: pass_scanBlocks(X); break;
    case WIG_PASS_SCAN_TOTALS: pass_scanTotals(X); break;
    case WIG_PASS_SCAN_FINISH: pass_scanFinish(X); break;
    case WIG_PASS_SCATTER: pass_scatter(X); break;
    case WIG_PASS_RASTER_CLAIMS: pass_rasterClaims(X); break;
    case WIG_PASS_RASTER: pass_raster(X); break;
    case WIG_PASS_UNPAINT: pass_unpaint(X); break;
    case WIG_PASS_BODY_START: pass_bodyStart(X); break;
    case WIG_PASS_BODY_LOADS: pass_bodyLoads(X); break;
    case WIG_PASS_BODY_DRAG: pass_bodyDrag(X); break;
    case WIG_PASS_BODY_FACES: pass_bodyFaces(X); break;
    case WIG_PASS_CG_BODY_X: pass_cgBodyX(X); break;
    case WIG_PASS_CG_BODY_P: pass_cgBodyP(X); break;
    case WIG_PASS_CG_BODY_F: pass_cgBodyF(X); break;
    case WIG_PASS_RIGIDIFY: pass_rigidify(X); break;
    case WIG_PASS_BODY_PUSH: pass_bodyPush(X); break;
    default: break;
    }
}

// The pressure operator of the FP64 solves: per fluid cell (in cell order)
// its four neighbours' rows and betas (fineBeta, the liquid neighbours
// only), its diagonal (the betas of every non-solid side, PIN at the root
// of a closed region) and the right-hand side -b.  With free bodies bound,
// the coupling J^T G J assembled on its own (fluid.wgsl:1374-1403, :2779-2795):
// per face from a fluid cell to a body's cell its J row (the normal and its
// arm about the body's centre, bodyFaceJ), and per body G, how it gives way
// (giveWay: the contact mobility worked out last step, else 1/m, 1/m, 1/I),
// so that (A p)_k = (L p)_k + sum over k's body faces of J . G (sum of J p).
struct F64System {
    struct Row { int32_t nb[4]; double beta[4]; double diag; };
    struct Couple { size_t k; uint32_t b; double j[3]; };
    std::vector<uint32_t> cellsOf;
    std::vector<Row> rows;
    std::vector<double> rhs;
    std::vector<Couple> couples;
    std::vector<std::array<double, 9>> give;  // per body, G row-major (bodies not coupled: unused)
    void couple(Ctx& X, size_t k, I2 c) {
        if (!X.motion) return;
        for (int dd = 0; dd < 4; dd++) {
            I2 q = Ctx::beside(c, dd);
            uint32_t b = rigidAt(X, q);
            if (b == NONE) continue;
            V3 j = bodyFaceJ(X, c, q, b);
            couples.push_back(Couple{k, b, {(double)j.x, (double)j.y, (double)j.z}});
            std::array<double, 9>& g = give[b];
            if (bodyWord(X, b, WIG_BW_MOBILITY_AT) != X.P->frame - 1u) {
                g = {1.0 / (double)rigidMass(X, b), 0, 0, 0, 1.0 / (double)rigidMass(X, b), 0, 0, 0,
                     1.0 / (double)rigidInertia(X, b)};
            } else {
                double m[6];
                for (uint32_t t = 0; t < 6; t++) m[t] = (double)bodyF(X, b, WIG_BW_MOBILITY + t);
                g = {m[0], m[1], m[2], m[1], m[3], m[4], m[2], m[4], m[5]};
            }
        }
    }
    size_t n() const { return cellsOf.size(); }
    void build(Ctx& X) {
        give.assign(X.motion ? MAX_BODIES : 0, std::array<double, 9>{});
        std::vector<int32_t> idx(X.C, -1);
        for (uint32_t i = 0; i < X.C; i++)
            if (X.fv(2u * i)[2] > 0.0f) { idx[i] = (int32_t)cellsOf.size(); cellsOf.push_back(i); }
        rows.resize(n());
        rhs.resize(n());
        for (size_t k = 0; k < n(); k++) {
            uint32_t i = cellsOf[k];
            I2 c{(int)(i % (uint32_t)X.W), (int)(i / (uint32_t)X.W)};
            float rho = X.fv(2u * i)[2];
            Row& r = rows[k];
            r.diag = 0.0;
            float share = X.shareAt(c);
            for (int dd = 0; dd < 4; dd++) {
                I2 nn = Ctx::beside(c, dd);
                r.nb[dd] = -1;
                r.beta[dd] = 0.0;
                float rr = rhoAt(X, 0, nn);
                if (rr < 0.0f) continue;
                double beta = (double)fineBeta(rho, rr, share, X.shareAt(nn));
                if (rr > 0.0f) { r.nb[dd] = idx[X.cellIndex(nn)]; r.beta[dd] = beta; }
                r.diag += beta;
            }
            if (pinnedAt(X, i)) r.diag += (double)PIN;
            rhs[k] = -(double)X.fv(2u * i)[1];
            couple(X, k, c);
        }
    }
    void apply(const std::vector<double>& p, std::vector<double>& q) const {
        for (size_t k = 0; k < n(); k++) {
            double s = rows[k].diag * p[k];
            for (int dd = 0; dd < 4; dd++)
                if (rows[k].nb[dd] >= 0) s -= rows[k].beta[dd] * p[rows[k].nb[dd]];
            q[k] = s;
        }
        if (couples.empty()) return;
        std::vector<std::array<double, 3>> jp(give.size(), std::array<double, 3>{0, 0, 0});
        for (const Couple& e : couples)
            for (int t = 0; t < 3; t++) jp[e.b][t] += e.j[t] * p[e.k];
        for (const Couple& e : couples) {
            const std::array<double, 9>& g = give[e.b];
            double v = 0.0;
            for (int t = 0; t < 3; t++) v += e.j[t] * (g[3 * t] * jp[e.b][0] + g[3 * t + 1] * jp[e.b][1] + g[3 * t + 2] * jp[e.b][2]);
            q[e.k] += v;
        }
    }
    void scatter(const std::vector<double>& x, uint32_t C, double* out) const {
        if (!out) return;
        for (uint32_t i = 0; i < C; i++) out[i] = 0.0;
        for (size_t k = 0; k < n(); k++) out[cellsOf[k]] = x[k];
    }
};

}  // namespace

// ---------------------------------------------------------------- C API of the oracle

extern "C" {

int wo_layout(const wig_world_desc* d, wig_world_layout* out) { return layout(d, out); }

// Binds the free bodies' host buffers for the passes and steps that follow
// (motion: WIG_BODY_MOTION_WORDS, pushes: WIG_MAX_BODIES * WIG_BODY_PUSH_WORDS
// u32; stamps: the bodies' buffer of the world, or null); motion and pushes
// null unbinds them all.
int wo_bind_bodies(uint32_t* motion, uint32_t* pushes, uint32_t* stamps) {
    if ((motion == nullptr) != (pushes == nullptr)) return WIG_E_ARG;
    g_motion = motion;
    g_pushes = pushes;
    g_stamps = motion ? stamps : nullptr;
    return WIG_OK;
}

// One pass (a reference pipeline dispatch) over host buffers.
int wo_pass(const wig_world_desc* d, const wig_params* P, const wig_elem* E, uint32_t nE, wig_fluid_buffers* b,
            int pass, uint32_t level, uint32_t cycle) {
    wig_world_layout L;
    int rc = layout(d, &L);
    if (rc) return rc;
    if (pass < 0 || pass >= WIG_PASS_COUNT) return WIG_E_ARG;
    Ctx X;
    setup(X, L, P, E, nE, b);
    X.level = level;
    X.cycle = cycle;
    run_pass(X, pass);
    return WIG_OK;
}

// One liquid step in encodeFluid's order (js/sim.js:2466-2612).  *shifted is
// the Simulation's shiftedFirst, toggled as the reference toggles it.
int wo_step(const wig_world_desc* d, const wig_params* P, const wig_elem* E, uint32_t nE, wig_fluid_buffers* b,
            uint32_t max_cycles, uint32_t flags, double tolerance, uint32_t* shifted, wig_fluid_stats* stats) {
    wig_world_layout L;
    int rc = layout(d, &L);
    if (rc) return rc;
    Ctx X;
    setup(X, L, P, E, nE, b);
    X.tol_mode = (flags & WIG_STEP_TOLERANCE) != 0u;
    X.f64_dots = (flags & WIG_STEP_F64_DOTS) != 0u;
    X.tol = tolerance;
    X.rel = 1.0;
    g_rz = g_pq = g_alpha = g_beta = 0.0;
    auto run = [&](int pass, uint32_t level = 0, uint32_t cycle = 0) {
        X.level = level;
        X.cycle = cycle;
        run_pass(X, pass);
    };
    if (flags & WIG_STEP_BOOKKEEPING_ONLY) {
        run(WIG_PASS_SYNC_MARKS);
        run(WIG_PASS_COMPACT);
        run(WIG_PASS_RETIRE);
    } else {
        run(WIG_PASS_SYNC);
        run(WIG_PASS_SYNC_PARTICLES);
        run(WIG_PASS_SYNC_SEED);
        run(WIG_PASS_COMPACT);
        run(WIG_PASS_RETIRE);
        run(WIG_PASS_CLEAR);
        run(WIG_PASS_GATHER);
        run(WIG_PASS_SEAL_JOIN);
        run(WIG_PASS_SEAL_ANCHOR);
        run(WIG_PASS_CLASSIFY);
        const bool bodies = X.motion != nullptr;
        if (bodies) { run(WIG_PASS_BODY_START); run(WIG_PASS_BODY_LOADS); }
        run(WIG_PASS_SET_FACES);
        if (flags & WIG_STEP_VISCOUS)
            for (int i = 0; i < 8; i++) { run(WIG_PASS_VISCOSITY_RED); run(WIG_PASS_VISCOSITY_BLACK); }
        run(WIG_PASS_UNPRESS);
        if (bodies && (flags & WIG_STEP_VISCOUS)) { run(WIG_PASS_BODY_DRAG); run(WIG_PASS_BODY_FACES); }
        run(WIG_PASS_DIVERGENCE);
        bool sh;
        if (flags & WIG_STEP_SHIFTED_SET) sh = (flags & WIG_STEP_SHIFTED_FIRST) != 0u;
        else { *shifted = *shifted ? 0u : 1u; sh = *shifted != 0u; }
        uint32_t deepest = L.levels;
        run(WIG_PASS_CG_START);
        run(WIG_PASS_CG_JOIN);
        run(WIG_PASS_CG_ANCHOR);
        if (bodies) run(WIG_PASS_CG_BODY_X);
        run(WIG_PASS_CG_RESIDUAL);
        run(WIG_PASS_CG_PREPARE);
        for (uint32_t cycle = 0; cycle < max_cycles; cycle++) {
            run(WIG_PASS_RELAX_RIMS, 0, cycle);
            run(sh ? WIG_PASS_RELAX_SHIFTED : WIG_PASS_RELAX, 0, cycle);
            sh = !sh;
            for (uint32_t l = 1; l <= deepest; l++) {
                run(WIG_PASS_RESTRICT, l, cycle);
                if (l < deepest) { run(WIG_PASS_SMOOTH_RED, l, cycle); run(WIG_PASS_SMOOTH_BLACK, l, cycle); }
            }
            run(WIG_PASS_SOLVE, deepest, cycle);
            for (uint32_t l = deepest - 1; l >= 1; l--) {
                run(WIG_PASS_PROLONG, l, cycle);
                run(WIG_PASS_SMOOTH_RED, l, cycle);
                run(WIG_PASS_SMOOTH_BLACK, l, cycle);
            }
            run(WIG_PASS_PROLONG_FINE, 0, cycle);
            run(WIG_PASS_RELAX_RIMS, 0, cycle);
            run(sh ? WIG_PASS_RELAX_SHIFTED : WIG_PASS_RELAX, 0, cycle);
            sh = !sh;
            run(WIG_PASS_CG_RHO, 0, cycle);
            run(WIG_PASS_CG_BETA, 0, cycle);
            run(WIG_PASS_CG_DIRECTION, 0, cycle);
            if (bodies) run(WIG_PASS_CG_BODY_P, 0, cycle);
            run(WIG_PASS_CG_APPLY, 0, cycle);
            run(WIG_PASS_CG_ALPHA, 0, cycle);
            run(WIG_PASS_CG_UPDATE, 0, cycle);
        }
        run(WIG_PASS_CG_FINISH);
        if (bodies) run(WIG_PASS_CG_BODY_F);
        run(WIG_PASS_PROJECT);
        if (bodies) { run(WIG_PASS_RIGIDIFY); run(WIG_PASS_BODY_PUSH); }
        run(WIG_PASS_EXTRAPOLATE);
        run(WIG_PASS_EXTRAPOLATE_FURTHER);
        run(WIG_PASS_ADVECT);
        run(WIG_PASS_SORT_COUNT);
        run(WIG_PASS_SCAN_BLOCKS);
        run(WIG_PASS_SCAN_TOTALS);
        run(WIG_PASS_SCAN_FINISH);
        run(WIG_PASS_SCATTER);
        run(WIG_PASS_RASTER_CLAIMS);
        run(WIG_PASS_RASTER);
        run(WIG_PASS_UNPAINT);
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        for (uint32_t k = 0; k < WIG_FLUID_STATS; k++) stats->count[k] = X.blocks[X.countSlot(k)];
        stats->particles = X.sorted[0];
        stats->cycles = X.blocks[X.countSlot(COUNT_CYCLES)];
        stats->rel_residual = X.rel;
        stats->b_norm = std::sqrt(X.bnorm2);
    }
    return WIG_OK;
}

// The FP64 reference solve: the same operator A (fineBeta, PIN at the roots
// of regions meeting no air) over the fluid cells as classify left them, the
// right-hand side -b (b the divergence in field's y), solved by CG with a
// Jacobi preconditioner in double to rel_tol.  Needs the step stopped after
// cgAnchor (the region links).  Writes x (per cell, 0 outside the liquid)
// and returns the iterations, or a negative code.
int wo_solve_f64(const wig_world_desc* d, const wig_params* P, const wig_elem* E, uint32_t nE, wig_fluid_buffers* b,
                 double rel_tol, uint32_t max_iter, double* x_out, double* rel_out) {
    wig_world_layout L;
    int rc = layout(d, &L);
    if (rc) return rc;
    Ctx X;
    setup(X, L, P, E, nE, b);
    F64System S;
    S.build(X);
    const size_t n = S.n();
    std::vector<double> x(n, 0.0), r(S.rhs), z(n), p(n), q(n);
    double bn = 0.0;
    for (double v : S.rhs) bn += v * v;
    bn = std::sqrt(bn);
    uint32_t it = 0;
    double rel = 0.0;
    if (bn > 0.0) {
        for (size_t k = 0; k < n; k++) z[k] = S.rows[k].diag > 0.0 ? r[k] / S.rows[k].diag : r[k];
        p = z;
        double rz = 0.0;
        for (size_t k = 0; k < n; k++) rz += r[k] * z[k];
        for (it = 0; it < max_iter; it++) {
            S.apply(p, q);
            double pq = 0.0;
            for (size_t k = 0; k < n; k++) pq += p[k] * q[k];
            if (pq <= 0.0) break;
            double a = rz / pq;
            double rr = 0.0;
            for (size_t k = 0; k < n; k++) { x[k] += a * p[k]; r[k] -= a * q[k]; rr += r[k] * r[k]; }
            rel = std::sqrt(rr) / bn;
            if (rel <= rel_tol) { it++; break; }
            double rz2 = 0.0;
            for (size_t k = 0; k < n; k++) { z[k] = S.rows[k].diag > 0.0 ? r[k] / S.rows[k].diag : r[k]; rz2 += r[k] * z[k]; }
            double beta = rz2 / rz;
            rz = rz2;
            for (size_t k = 0; k < n; k++) p[k] = z[k] + beta * p[k];
        }
    }
    S.scatter(x, X.C, x_out);
    if (rel_out) *rel_out = rel;
    return (int)it;
}

// The same FP64 solve (operator, right-hand side, output) with one V-cycle
// of this oracle's own FP32 passes as the preconditioner, for worlds where
// the Jacobi form needs thousands of iterations (2048 x 2048).  The outer
// iteration is flexible CG in double: beta = -(z . q_prev) / (p_prev . q_prev)
// (the reference's flexible beta, fluid.wgsl:2752-2764), alpha = (p . r) /
// (p . q), every vector, dot product and residual FP64.  The preconditioner
// puts r, scaled to a largest entry of 1, into field's right-hand sides
// (-r, as cgPrepare and cgUpdate leave them, fluid.wgsl:2721-2732,
// :2852-2880), zeroes the potentials, runs relaxRims, relax, restrict and
// smooth down the levels, solve, prolong and smooth up, prolongFine,
// relaxRims, relax (encodeFluid's cycle, js/sim.js:2557-2588), and reads z
// back from the potentials.  Its FP32 rounding bounds how much one
// iteration gains, not the accuracy reached: the residual is FP64 and the
// solve runs to rel_tol.  The buffers hold the V-cycle's scratch afterwards
// (potentials, coarse levels, rims), so callers solve on a copy.
int wo_solve_f64_mg(const wig_world_desc* d, const wig_params* P, const wig_elem* E, uint32_t nE, wig_fluid_buffers* b,
                    double rel_tol, uint32_t max_iter, double* x_out, double* rel_out) {
    wig_world_layout L;
    int rc = layout(d, &L);
    if (rc) return rc;
    Ctx X;
    setup(X, L, P, E, nE, b);
    F64System S;
    S.build(X);
    const size_t n = S.n();
    // every pass of the cycle runs: the tolerance form's test with rel above tol
    X.tol_mode = true;
    X.tol = 0.0;
    X.rel = 1.0;
    X.cycle = 0;
    bool sh = false;
    auto vcycle = [&](const std::vector<double>& r, std::vector<double>& z) {
        double scale = 0.0;
        for (double v : r) scale = wmax(scale, std::fabs(v));
        if (scale == 0.0) scale = 1.0;
        for (uint32_t i = 0; i < X.C; i++) X.fv(2u * i)[0] = 0.0f;
        for (size_t k = 0; k < n; k++) X.fv(2u * S.cellsOf[k])[1] = (float)(-r[k] / scale);
        auto run = [&](int pass, uint32_t level) { X.level = level; run_pass(X, pass); };
        const uint32_t deepest = L.levels;
        run(WIG_PASS_RELAX_RIMS, 0);
        run(sh ? WIG_PASS_RELAX_SHIFTED : WIG_PASS_RELAX, 0);
        sh = !sh;
        for (uint32_t l = 1; l <= deepest; l++) {
            run(WIG_PASS_RESTRICT, l);
            if (l < deepest) { run(WIG_PASS_SMOOTH_RED, l); run(WIG_PASS_SMOOTH_BLACK, l); }
        }
        run(WIG_PASS_SOLVE, deepest);
        for (uint32_t l = deepest - 1; l >= 1; l--) {
            run(WIG_PASS_PROLONG, l);
            run(WIG_PASS_SMOOTH_RED, l);
            run(WIG_PASS_SMOOTH_BLACK, l);
        }
        run(WIG_PASS_PROLONG_FINE, 0);
        run(WIG_PASS_RELAX_RIMS, 0);
        run(sh ? WIG_PASS_RELAX_SHIFTED : WIG_PASS_RELAX, 0);
        sh = !sh;
        for (size_t k = 0; k < n; k++) z[k] = scale * (double)X.fv(2u * S.cellsOf[k])[0];
    };
    auto dot = [&](const std::vector<double>& a, const std::vector<double>& c) {
        double s = 0.0;
        for (size_t k = 0; k < n; k++) s += a[k] * c[k];
        return s;
    };
    std::vector<double> x(n, 0.0), r(S.rhs), z(n), p(n, 0.0), q(n, 0.0);
    const double bn = std::sqrt(dot(S.rhs, S.rhs));
    uint32_t it = 0;
    double rel = bn > 0.0 ? 1.0 : 0.0, pq_prev = 0.0;
    if (bn > 0.0) {
        for (it = 0; it < max_iter; it++) {
            vcycle(r, z);
            const double beta = (it == 0 || pq_prev <= 0.0) ? 0.0 : -dot(z, q) / pq_prev;
            for (size_t k = 0; k < n; k++) p[k] = z[k] + beta * p[k];
            S.apply(p, q);
            const double pq = dot(p, q);
            if (pq <= 0.0) break;
            const double a = dot(p, r) / pq;
            double rr = 0.0;
            for (size_t k = 0; k < n; k++) { x[k] += a * p[k]; r[k] -= a * q[k]; rr += r[k] * r[k]; }
            pq_prev = pq;
            rel = std::sqrt(rr) / bn;
            if (rel <= rel_tol) { it++; break; }
        }
    }
    S.scatter(x, X.C, x_out);
    if (rel_out) *rel_out = rel;
    return (int)it;
}

// ||-b - A x||2 / ||b||2 in FP64 for a pressure x (per cell, as f32), the
// operator as in wo_solve_f64.
double wo_true_residual(const wig_world_desc* d, const wig_params* P, const wig_elem* E, uint32_t nE,
                        wig_fluid_buffers* b, const float* x) {
    wig_world_layout L;
    if (layout(d, &L)) return -1.0;
    Ctx X;
    setup(X, L, P, E, nE, b);
    double rr = 0.0, bb = 0.0;
    for (uint32_t i = 0; i < X.C; i++) {
        float rho = X.fv(2u * i)[2];
        if (rho <= 0.0f) continue;
        I2 c{(int)(i % (uint32_t)X.W), (int)(i / (uint32_t)X.W)};
        float share = X.shareAt(c);
        double diag = 0.0, s = 0.0;
        for (int dd = 0; dd < 4; dd++) {
            I2 nn = Ctx::beside(c, dd);
            float rr2 = rhoAt(X, 0, nn);
            if (rr2 < 0.0f) continue;
            double beta = (double)fineBeta(rho, rr2, share, X.shareAt(nn));
            if (rr2 > 0.0f) s += beta * (double)x[X.cellIndex(nn)];
            diag += beta;
        }
        if (pinnedAt(X, i)) diag += (double)PIN;
        double bi = (double)X.fv(2u * i)[1];
        double ri = -bi - (diag * (double)x[i] - s);
        rr += ri * ri;
        bb += bi * bi;
    }
    return bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
}

// sin/cos of the own implementation, for the tests to compare with.
void wo_sincos(float a, float* s, float* c) { sincos_own(a, s, c); }

// exactParts and exactValue (common.wgsl:1378-1412) at EXACT_COARSE, the
// scale of the bodies' push sums, for the tests of their two-word sums.
void wo_exact_parts(float x, uint32_t* lo, uint32_t* hi) { exactParts(x, EXACT_COARSE, lo, hi); }
float wo_exact_value(uint32_t lo, uint32_t hi) { return exactValue(lo, hi, EXACT_COARSE); }

}  // extern "C"
