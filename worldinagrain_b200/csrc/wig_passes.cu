// wig_passes.cu — the liquid step's passes as sm_100a kernels, one per
// pipeline that Simulation.encodeFluid dispatches (js/sim.js:2466-2612), over
// the reference's buffer layouts.  Each kernel cites the WGSL entry point it
// replaces.  Grid shapes: the passes over the blocks worked on run one CTA of
// 64 threads (8 x 8 cells) per block, grid-striding over the active list, so
// the launch is sized to the device (148 SMs) rather than to the world; the
// passes over particles run a thread per live particle; the coarse levels a
// thread per coarse cell.
//
// Arithmetic: this file is compiled with --fmad=false and IEEE division and
// square root, so each f32 operation rounds on its own as in the WGSL, and
// every reduction runs in a fixed tree order (the reference's block-index
// order, fluid.wgsl:2538-2542).  The grid buffers it leaves are bit-for-bit
// those of a sequential restatement; only the order of particles within a
// cell's run depends on thread timing, as in the reference (sortCount's slot
// is an atomic's order, fluid.wgsl:3707).

#include "wig_device.cuh"
#include "wig_passes.cuh"

namespace wig {

// ---------------------------------------------------------------- helpers

// The blocks worked on, grid-strided: wid over [0, activeCount).
#define FOR_ACTIVE(D, w, wid)                                      \
    const uint32_t n_active_ = (w).activeCount();                  \
    for (uint32_t wid = blockIdx.x; wid < n_active_; wid += gridDim.x)

__device__ __forceinline__ I2 lidCell(const W& w, uint32_t wid) {
    I2 b = w.activeBlock(wid);
    return I2{b.x * BLOCK + (int)(threadIdx.x & 7u), b.y * BLOCK + (int)(threadIdx.x >> 3)};
}

__device__ __forceinline__ uint32_t vload(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// union-find over G_REGION words (label.wgsl:27-55), lock-free by atomicMin.
__device__ uint32_t ufFind(const W& w, uint32_t i) {
    uint32_t x = i;
    const uint32_t limit = g_loop_limit;
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t up = vload(w.gwp(x, G_REGION));
        if (up >= x) return x;
        x = up;
    }
    atomicOr(&w.D.st->err, ERR_LOOP);
    return x;
}
__device__ void ufJoin(const W& w, uint32_t i, uint32_t j) {
    uint32_t a = i, b = j;
    const uint32_t limit = g_loop_limit;
    for (uint32_t it = 0; it < limit; it++) {
        a = ufFind(w, a);
        b = ufFind(w, b);
        if (a == b) return;
        uint32_t lo = min(a, b), hi = max(a, b);
        uint32_t old = atomicMin(w.gwp(hi, G_REGION), lo);
        if (old == hi) return;
        a = old;
        b = lo;
    }
    atomicOr(&w.D.st->err, ERR_LOOP);
}
__device__ __forceinline__ bool pinnedAt(const W& w, uint32_t i) { return vload(w.gwp(i, G_REGION)) == i; }

// isObstacleCell, countAt, liquidIn (fluid.wgsl:1120-1179)
__device__ bool isLiquidAt(const W& w, I2 c) { return w.inWorld(c) && w.kindOfCell(w.cellIndex(c)) == WIG_KIND_LIQUID; }
__device__ bool fallingAt(const W& w, I2 q) {
    if (!w.inWorld(q)) return false;
    uint32_t fb = 4u << ((w.D.st->P.frame + 1u) & 1u);
    return (f2u(w.fv(2u * w.cellIndex(q) + 1u)[3]) & fb) != 0u;
}
__device__ bool isObstacleCell(const W& w, I2 c) {
    uint32_t i = w.cellIndex(c);
    uint32_t t = w.cellType(i);
    uint32_t k = w.kindOf(t);
    if (k == WIG_KIND_GAS) {
        int wet = 0;
        for (int d = 0; d < 4; d++) wet += isLiquidAt(w, beside(c, d)) ? 1 : 0;
        if (wet < 2) return false;
        if (t == AIR) {
            I2 up1{c.x, c.y - 1}, up2{c.x, c.y - 2};
            if (!isLiquidAt(w, up1) || !isLiquidAt(w, up2) || fallingAt(w, up1)) return false;
            return w.gasAmountOf(i) >= BUBBLE_GAS;
        }
        return true;
    }
    return k == WIG_KIND_SOLID || k == WIG_KIND_POWDER;
}
__device__ int countAt(const W& w, I2 c) {
    if (!w.inWorld(c)) return -1;
    if (isObstacleCell(w, c)) return -1;
    return (int32_t)w.gw(w.cellIndex(c), G_COUNT);
}
__device__ V2 liquidIn(const W& w, uint32_t i) {
    uint4 v = w.cell(i);
    uint32_t t = wordType(v.x);
    const wig_elem& e = w.elem(t);
    float temp = __uint_as_float(v.y);
    float acts = w.actsAt(v.x, temp);
    float viscosity = e.kind == WIG_KIND_LIQUID ? w.viscosityAt(e, acts) : 0.0f;
    uint32_t n = w.gw(i, G_COUNT);
    if (n > 0u) return V2{(float)w.gw(i, G_MASS) / (FIX * (float)n), viscosity};
    if (e.kind != WIG_KIND_LIQUID) return V2{1.0f, 0.0f};
    return V2{w.liquidDensity(v.x, temp), viscosity};
}

// ---------------------------------------------------------------- levels
__device__ __forceinline__ I2 levelSize(const Dev& D, uint32_t l) { return I2{(int)D.level_w[l], (int)D.level_h[l]}; }
__device__ __forceinline__ bool inLevel(const Dev& D, uint32_t l, I2 c) {
    return c.x >= 0 && c.y >= 0 && c.x < (int)D.level_w[l] && c.y < (int)D.level_h[l];
}
__device__ __forceinline__ uint32_t levelSlot(const Dev& D, uint32_t l, I2 c) {
    return D.level_start[l] + 2u * ((uint32_t)c.y * D.level_w[l] + (uint32_t)c.x);
}
__device__ __forceinline__ float rhoAt(const W& w, uint32_t l, I2 c) {
    if (!inLevel(w.D, l, c)) return -1.0f;
    if (l == 0u) return w.fv(2u * w.cellIndex(c))[2];
    return w.fv(levelSlot(w.D, l, c) + 1u)[0];
}
__device__ __forceinline__ V2 potAt(const W& w, uint32_t l, I2 c) {
    if (!inLevel(w.D, l, c)) return V2{0.0f, 0.0f};
    if (l == 0u) {
        uint32_t i = 2u * w.cellIndex(c);
        return V2{w.fv(i)[0], w.fv(i + 1u)[0]};
    }
    float* f = w.fv(levelSlot(w.D, l, c));
    return V2{f[0], f[1]};
}
__device__ __forceinline__ V2 rhsAt(const W& w, uint32_t l, I2 c) {
    if (l == 0u) {
        uint32_t i = 2u * w.cellIndex(c);
        return V2{w.fv(i)[1], w.fv(i + 1u)[1]};
    }
    float* f = w.fv(levelSlot(w.D, l, c));
    return V2{f[2], f[3]};
}
// stencil (fluid.wgsl:2286-2302)
__device__ void stencil(const W& w, uint32_t l, I2 c, float rho, V2* sum, float* diag) {
    V2 s{0.0f, 0.0f};
    float dg = 0.0f;
    for (int d = 0; d < 4; d++) {
        I2 n = beside(c, d);
        float r = rhoAt(w, l, n);
        if (r < 0.0f) continue;
        float beta = faceBeta(rho, r);
        if (l == 0u) beta = fineBeta(rho, r, w.densityAt(c), w.densityAt(n));
        V2 p = potAt(w, l, n);
        s.x = s.x + beta * p.x;
        s.y = s.y + beta * p.y;
        dg = dg + beta;
    }
    *sum = s;
    *diag = dg;
}
// residualAt (fluid.wgsl:2306-2315)
__device__ V2 residualAt(const W& w, uint32_t l, I2 c) {
    float rho = rhoAt(w, l, c);
    if (rho <= 0.0f) return V2{0.0f, 0.0f};
    V2 sum;
    float diag;
    stencil(w, l, c, rho, &sum, &diag);
    float h2 = (float)(1u << (2u * l));
    float pinx = (l == 0u && pinnedAt(w, w.cellIndex(c))) ? PIN : 0.0f;
    V2 p = potAt(w, l, c), rhs = rhsAt(w, l, c);
    return V2{rhs.x - (sum.x - (diag + pinx) * p.x) / h2, rhs.y - (sum.y - (diag + 0.0f) * p.y) / h2};
}
// prolonged (fluid.wgsl:2478-2497)
__device__ V2 prolonged(const W& w, uint32_t l, I2 c) {
    I2 coarse{c.x / 2, c.y / 2};
    int sx = (c.x & 1) == 1 ? 1 : -1, sy = (c.y & 1) == 1 ? 1 : -1;
    const int ox[4] = {0, sx, 0, sx}, oy[4] = {0, 0, sy, sy};
    const float wt[4] = {9.0f, 3.0f, 3.0f, 1.0f};
    V2 sum{0.0f, 0.0f};
    float weight = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        I2 at{coarse.x + ox[k], coarse.y + oy[k]};
        float r = rhoAt(w, l + 1u, at);
        if (r < 0.0f) continue;
        weight = weight + wt[k];
        if (r > 0.0f) {
            V2 p = potAt(w, l + 1u, at);
            sum.x = sum.x + wt[k] * p.x;
            sum.y = sum.y + wt[k] * p.y;
        }
    }
    float ww = fmaxf(weight, 1e-6f);
    return V2{sum.x / ww, sum.y / ww};
}

// ================================================================ free bodies
// (fluid.wgsl:1181-1470; the body table's words, js/shared.js:294-333).  The
// pushes are exact two-word sums (common.wgsl:1378-1412) added by atomics, so
// their totals do not depend on the order the cells add them in.

constexpr uint32_t MAX_BODIES = WIG_MAX_BODIES;
constexpr uint32_t PUSH_P0 = 0, PUSH_X = 2, PUSH_F = 3, PUSH_SURFACE = 4, PUSH_DRAG = 5;
constexpr float EXACT_COARSE = 16777216.0f;
constexpr int SEEP_REACH = 128;
struct V3 { float x, y, z; };

__device__ __forceinline__ uint32_t bodyWord(const W& w, uint32_t b, uint32_t k) {
    return w.D.motion[MAX_BODIES + b * WIG_BODY_TABLE_WORDS + k];
}
__device__ __forceinline__ float bodyF(const W& w, uint32_t b, uint32_t k) { return __uint_as_float(bodyWord(w, b, k)); }
__device__ __forceinline__ V2 bodyV(const W& w, uint32_t b, uint32_t k) { return V2{bodyF(w, b, k), bodyF(w, b, k + 1u)}; }
__device__ __forceinline__ uint32_t liquidSlot(uint32_t b, uint32_t k) { return WIG_BODY_LIQUID_BASE + b * WIG_BODY_LIQUID_WORDS + k; }
__device__ __forceinline__ bool bodyInSolve(const W& w, uint32_t b) {
    uint32_t flags = bodyWord(w, b, WIG_BW_FLAGS);
    return !((flags & WIG_BF_ALIVE) == 0u || (flags & WIG_BF_NEW) != 0u || bodyF(w, b, WIG_BW_MASS) <= 0.0f);
}
// rigidBodyOf (fluid.wgsl:1233-1248)
__device__ uint32_t rigidBodyOf(const W& w, uint4 v) {
    const uint32_t t = wordType(v.x);
    const wig_elem& e = w.elem(t);
    if (!wordHas(v.x, WIG_FL_LOOSE) || e.kind != WIG_KIND_SOLID || e.break_to == WIG_NO_ELEM) return NONE;
    const float id = f16_value(v.w & 0xffffu);
    if (id < 0.0f || id >= (float)MAX_BODIES) return NONE;
    const uint32_t b = f2u(id);
    return bodyInSolve(w, b) ? b : NONE;
}
__device__ __forceinline__ float rigidMass(const W& w, uint32_t b) { return bodyF(w, b, WIG_BW_MASS) + bodyF(w, b, WIG_BW_CARGO); }
__device__ __forceinline__ float rigidInertia(const W& w, uint32_t b) {
    return bodyF(w, b, WIG_BW_INERTIA) + bodyF(w, b, WIG_BW_CARGO_INERTIA);
}
__device__ __forceinline__ float bodyDensity(const W& w, uint32_t b) {
    return rigidMass(w, b) / fmaxf((float)bodyWord(w, b, WIG_BW_CELLS), 1.0f);
}
__device__ __forceinline__ bool isHeld(const W& w, uint32_t b) { return (bodyWord(w, b, WIG_BW_FLAGS) & WIG_BF_HELD) != 0u; }
// wetRegionAt (fluid.wgsl:592-595)
__device__ bool wetRegionAt(const W& w, uint4 v) {
    if (!w.D.motion) return false;
    const uint32_t b = rigidBodyOf(w, v);
    return b != NONE && (bodyWord(w, b, WIG_BW_FLAGS) & (WIG_BF_WET | WIG_BF_HELD)) == (WIG_BF_WET | WIG_BF_HELD);
}
// bodySweptSlot, claimStep (common.wgsl:316-385): cell i's stamp of step frame
__device__ __forceinline__ uint32_t claimStep(uint32_t frame) { return frame % WIG_CLAIM_PERIOD + 1u; }
__device__ __forceinline__ uint32_t bodySweptSlot(const W& w, uint32_t i, uint32_t frame) {
    const uint32_t tiles = (((uint32_t)w.D.W + WIG_BODY_TILE - 1u) / WIG_BODY_TILE) *
                           (((uint32_t)w.D.H + WIG_BODY_TILE - 1u) / WIG_BODY_TILE);
    const uint32_t base = 4u * tiles + WIG_BODY_STAT_WORDS + WIG_BODY_COUNTERS + MAX_BODIES + (2u + WIG_BODY_SUM_WORDS) * w.D.C;
    return base + 1u + tiles + 2u * w.D.C + w.D.C + 2u * i + (frame & 1u);
}
// cupOf, seamOf (fluid.wgsl:1252-1288): the body whose cup (seam) cell i was
// stamped last step, alive and weighed; cupBefore (fluid.wgsl:3521-3528):
// whose cup it was the step before, whatever the body's state now
__device__ uint32_t sweptBody(const W& w, uint32_t i, uint32_t frame, uint32_t seam) {
    if (!w.D.stamps || !w.D.motion) return NONE;
    const uint32_t key = w.D.stamps[bodySweptSlot(w, i, frame)];
    if ((key >> 12u) != claimStep(frame) || (key & 1u) != seam) return NONE;
    const uint32_t b = 2047u - ((key >> 1u) & 0x7ffu);
    return b < MAX_BODIES ? b : NONE;
}
__device__ uint32_t cupOf(const W& w, uint32_t i) {
    const uint32_t b = sweptBody(w, i, w.D.st->P.frame - 1u, 0u);
    return b != NONE && bodyInSolve(w, b) ? b : NONE;
}
__device__ uint32_t seamOf(const W& w, uint32_t i) {
    const uint32_t b = sweptBody(w, i, w.D.st->P.frame - 1u, 1u);
    return b != NONE && bodyInSolve(w, b) ? b : NONE;
}
__device__ __forceinline__ uint32_t cupBefore(const W& w, uint32_t i) { return sweptBody(w, i, w.D.st->P.frame - 2u, 0u); }
// rigidAt, heldAt (fluid.wgsl:1422-1458): the body classify put in the drift's z
__device__ uint32_t rigidAt(const W& w, I2 c) {
    if (!w.D.motion || !w.inWorld(c)) return NONE;
    const float z = w.fv(2u * w.cellIndex(c) + 1u)[2];
    const uint32_t b = f2u(fmaxf(-z, 1.0f)) - 1u;
    return (z < 0.0f && b < MAX_BODIES) ? b : NONE;
}
__device__ uint32_t heldAt(const W& w, I2 c) {
    if (!w.D.motion || !w.inWorld(c)) return NONE;
    const float z = w.fv(2u * w.cellIndex(c) + 1u)[2];
    const uint32_t b = f2u(fmaxf(-z, 1.0f)) - 1u;
    // (a slot past the table, from a drift word classify did not write, is none)
    return (z < 0.0f && b >= MAX_BODIES && b < 2u * MAX_BODIES) ? b - MAX_BODIES : NONE;
}
// exactParts, exactValue (common.wgsl:1378-1412)
__device__ __forceinline__ void exactParts(float x, float scale, uint32_t* lo, uint32_t* hi) {
    const float s = rnd_even(clampf(x * scale, -9.2e18f, 9.2e18f));
    if (fabsf(s) < 2147483648.0f) {
        const int32_t v = f2i(s);
        *lo = (uint32_t)v;
        *hi = v < 0 ? 0xffffffffu : 0u;
        return;
    }
    const float h = floorf(s / 4294967296.0f);
    *lo = f2u(s - h * 4294967296.0f);
    *hi = (uint32_t)f2i(h);
}
__device__ __forceinline__ float exactValue(uint32_t lo, uint32_t hi, float scale) {
    const int32_t l = (int32_t)lo, h = (int32_t)hi;
    if ((h == 0 && l >= 0) || (h == -1 && l < 0)) return __int2float_rn(l) / scale;
    return (__int2float_rn(h) * 4294967296.0f + __uint2float_rn(lo)) / scale;
}
// pushSlot, addPush, pushOf (fluid.wgsl:1318-1338)
__device__ __forceinline__ uint32_t pushSlot(uint32_t b, uint32_t which, uint32_t k) {
    return b * WIG_BODY_PUSH_WORDS + 6u * which + 2u * k;
}
__device__ void addPush(const W& w, uint32_t b, uint32_t which, V3 v) {
    const float c[3] = {v.x, v.y, v.z};
    for (uint32_t k = 0; k < 3; k++) {
        uint32_t lo, hi;
        exactParts(c[k], EXACT_COARSE, &lo, &hi);
        uint32_t* at = w.D.pushes + pushSlot(b, which, k);
        const uint32_t old = atomicAdd(at, lo);
        atomicAdd(at + 1, hi + (old + lo < old ? 1u : 0u));
    }
}
__device__ V3 pushOf(const W& w, uint32_t b, uint32_t which) {
    const uint32_t* at = w.D.pushes + pushSlot(b, which, 0u);
    return V3{exactValue(at[0], at[1], EXACT_COARSE), exactValue(at[2], at[3], EXACT_COARSE),
              exactValue(at[4], at[5], EXACT_COARSE)};
}
// giveWay, pushChange, pushChangeFree (fluid.wgsl:1348-1372)
__device__ V3 giveWay(const W& w, uint32_t b, V3 g) {
    if (bodyWord(w, b, WIG_BW_MOBILITY_AT) != w.D.st->P.frame - 1u)
        return V3{g.x / rigidMass(w, b), g.y / rigidMass(w, b), g.z / rigidInertia(w, b)};
    float m[6];
    for (uint32_t k = 0; k < 6; k++) m[k] = bodyF(w, b, WIG_BW_MOBILITY + k);
    return V3{m[0] * g.x + m[1] * g.y + m[2] * g.z, m[1] * g.x + m[3] * g.y + m[4] * g.z,
              m[2] * g.x + m[4] * g.y + m[5] * g.z};
}
__device__ __forceinline__ V3 pushChange(const W& w, uint32_t b, uint32_t which) { return giveWay(w, b, pushOf(w, b, which)); }
__device__ V3 pushChangeFree(const W& w, uint32_t b, uint32_t which) {
    const V3 g = pushOf(w, b, which);
    return V3{g.x / rigidMass(w, b), g.y / rigidMass(w, b), g.z / rigidInertia(w, b)};
}
// bodyFaceJ (fluid.wgsl:1374-1379): the face from cell c to body b's cell q
__device__ V3 bodyFaceJ(const W& w, I2 c, I2 q, uint32_t b) {
    const V2 n{(float)(q.x - c.x), (float)(q.y - c.y)};
    const V2 pos = bodyV(w, b, WIG_BW_POS);
    const V2 r{(((float)c.x + 0.5f) + 0.5f * n.x) - pos.x, (((float)c.y + 0.5f) + 0.5f * n.y) - pos.y};
    return V3{n.x, n.y, r.x * n.y - r.y * n.x};
}
__device__ __forceinline__ V3 scale3(V3 v, float s) { return V3{v.x * s, v.y * s, v.z * s}; }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// addPressurePush, couplingAt (fluid.wgsl:1381-1403)
__device__ void addPressurePush(const W& w, I2 c, float p, uint32_t which) {
    for (int d = 0; d < 4; d++) {
        const I2 q = beside(c, d);
        const uint32_t b = rigidAt(w, q);
        if (b != NONE) addPush(w, b, which, scale3(bodyFaceJ(w, c, q, b), p));
    }
}
__device__ float couplingAt(const W& w, I2 c, uint32_t which) {
    float sum = 0.0f;
    if (!w.D.motion) return sum;
    for (int d = 0; d < 4; d++) {
        const I2 q = beside(c, d);
        const uint32_t b = rigidAt(w, q);
        if (b != NONE) sum = sum + dot3(bodyFaceJ(w, c, q, b), pushChange(w, b, which));
    }
    return sum;
}
// rigidVel (fluid.wgsl:1460-1465), bodyMoving (fluid.wgsl:1410-1419)
__device__ V2 rigidVel(const W& w, uint32_t b, V2 x) {
    const V2 pos = bodyV(w, b, WIG_BW_POS);
    const V2 r{x.x - pos.x, x.y - pos.y};
    const float spin = bodyF(w, b, WIG_BW_SPIN);
    const V2 v = bodyV(w, b, WIG_BW_VEL);
    return V2{v.x + -spin * r.y, v.y + spin * r.x};
}
__device__ V2 bodyMoving(const W& w, uint32_t b, V2 x, bool drag) {
    const V2 pos = bodyV(w, b, WIG_BW_POS);
    const V2 pull = w.pull();
    const float m = rigidMass(w, b);
    V3 ch = add3(pushChange(w, b, PUSH_SURFACE), giveWay(w, b, V3{m * pull.x, m * pull.y, 0.0f}));
    if (drag) ch = add3(ch, pushChange(w, b, PUSH_DRAG));
    const V2 r{x.x - pos.x, x.y - pos.y};
    const V2 rv = rigidVel(w, b, x);
    const V2 px = w.pull();
    return V2{(((rv.x + px.x) - pull.x) + ch.x) + -ch.z * r.y, (((rv.y + px.y) - pull.y) + ch.y) + ch.z * r.x};
}
// bodyReach (fluid.wgsl:413-415)
__device__ float bodyReach(const W& w, uint32_t b, I2 n) {
    const uint32_t s = bodyWord(w, b, WIG_BW_SUBCELL);
    const float sx = f16_value(s & 0xffffu), sy = f16_value(s >> 16);
    return clampf(0.5f + (sx * (float)n.x + sy * (float)n.y), 0.0f, 1.0f);
}
// posedRoom (fluid.wgsl:2035-2045)
__device__ float posedRoom(const W& w, I2 c) {
    float room = 1.0f;
    for (int d = 0; d < 4; d++) {
        const I2 q = beside(c, d);
        const uint32_t b = rigidAt(w, q);
        if (b != NONE) room = room + (0.5f - bodyReach(w, b, I2{c.x - q.x, c.y - q.y}));
    }
    return clampf(room, 0.1f, 1.9f);
}
// faceMiddle (fluid.wgsl:1473-1475)
__device__ __forceinline__ V2 faceMiddle(I2 at, bool isU) {
    return isU ? V2{(float)at.x + 0.0f, (float)at.y + 0.5f} : V2{(float)at.x + 0.5f, (float)at.y + 0.0f};
}
// potentialAt (fluid.wgsl:2958-2960): the masses' potential none (binding 10 unbound)
__device__ __forceinline__ float potentialAt(const W& w, V2 pos) {
    return w.D.st->P.earth_g * ((float)w.D.H - pos.y) + 0.0f;
}
// seepAt (fluid.wgsl:2977-3000)
__device__ float seepAt(const W& w, I2 c, I2 n, uint32_t h, bool held, V2 x) {
    I2 ways[2] = {I2{-1, 0}, I2{1, 0}};
    int count = 2;
    if (n.x != 0) {
        ways[0] = I2{-n.x, -n.y};
        count = 1;
    }
    int nearest = SEEP_REACH + 1;
    float p = 0.0f;
    for (int k2 = 0; k2 < count; k2++) {
        for (int k = 1; k < nearest; k++) {
            const I2 q{c.x + ways[k2].x * k, c.y + ways[k2].y * k};
            if ((held ? heldAt(w, q) : rigidAt(w, q)) == h) continue;
            const float4 g = w.gridAt(q);
            if (g.z > 0.0f) {
                nearest = k;
                p = g.x + g.z * (potentialAt(w, V2{(float)q.x + 0.5f, (float)q.y + 0.5f}) - potentialAt(w, x));
            }
            break;
        }
    }
    return p;
}
// heldPush (fluid.wgsl:3007-3031)
__device__ void heldPush(const W& w, I2 c, uint32_t h, int32_t out[3]) {
    const V2 pos = bodyV(w, h, WIG_BW_POS);
    V2 f{0.0f, 0.0f};
    float torque = 0.0f;
    for (int d = 0; d < 4; d++) {
        const I2 q = beside(c, d);
        const I2 n{q.x - c.x, q.y - c.y};
        if (heldAt(w, q) == h) continue;
        const float4 g = w.gridAt(q);
        const V2 x{((float)c.x + 0.5f) + 0.5f * (float)n.x, ((float)c.y + 0.5f) + 0.5f * (float)n.y};
        float p = g.x;
        if (g.z > 0.0f) p = p + g.z * (potentialAt(w, V2{(float)q.x + 0.5f, (float)q.y + 0.5f}) - potentialAt(w, x));
        else if (g.z < 0.0f) p = seepAt(w, c, n, h, true, x);
        const V2 push{-p * (float)n.x, -p * (float)n.y};
        f = V2{f.x + push.x, f.y + push.y};
        const V2 r{x.x - pos.x, x.y - pos.y};
        torque = torque + (r.x * push.y - r.y * push.x);
    }
    out[0] = f2i(rnd_even((f.x / rigidMass(w, h)) * WIG_RIGID_FIX));
    out[1] = f2i(rnd_even((f.y / rigidMass(w, h)) * WIG_RIGID_FIX));
    out[2] = f2i(rnd_even((torque / rigidInertia(w, h)) * WIG_RIGID_FIX));
}

// ================================================================ bookkeeping

// sync / syncMarks (fluid.wgsl:608-659): a CTA per block of the world
// (syncMarks: no claims, as a world's bookkeeping-only step takes it).
__global__ void k_sync(Batch Bt, int sync_claims) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
  FOR_ITEMS(Bt, L_WB, it) {
    ITEM_WORLD_C(Bt, it, D, w, n);
    const bool claims = sync_claims && D.st->book == 0u;
    const I2 b = w.blockAt(n);
    I2 c{b.x * BLOCK + (int)(threadIdx.x & 7u), b.y * BLOCK + (int)(threadIdx.x >> 3)};
    bool here = false, region = false;
    if (w.inWorld(c)) {
        uint32_t i = w.cellIndex(c);
        if (i == 0u) {
            D.parts[0] = 0u;
            D.blocks[w.countSlot(COUNT_ACTIVE)] = 0u;
            D.blocks[w.countSlot(COUNT_RETIRED)] = 0u;
            D.blocks[w.countSlot(COUNT_VISCOUS)] = 0u;
        }
        uint4 v = w.cell(i);
        if (w.kindOf(wordType(v.x)) == WIG_KIND_LIQUID) {
            uint32_t home = liquidHome(v.w);
            if (claims && wordHas(v.x, FL_DRAWN) && home < D.C) atomicMax(w.gwp(home, G_DEST), claimOf(i));
            here = true;
        } else if (wetRegionAt(w, v)) {
            region = true;
        }
    }
    if (__syncthreads_or(here) && threadIdx.x == 0) atomicOr(&D.blocks[n], MARK_LIQUID);
    if (__syncthreads_or(region) && threadIdx.x == 0) atomicOr(&D.blocks[n], MARK_REGION);
  }
}

__device__ void markBlockOf(const W& w, float px, float py) {
    I2 c = w.cellOf(px, py);
    I2 b{c.x / BLOCK, c.y / BLOCK};
    if (w.inBlocks(b)) atomicOr(&w.D.blocks[w.blockIndex(b)], MARK_LIQUID);
}

__device__ V2 pairWay(uint32_t a, uint32_t b) {
    uint32_t h = pcg(min(a, b) ^ pcg(max(a, b)));
    float angle = (float)h * (float)(6.2831853 / 4294967296.0);
    float s, c;
    sincos_own(angle, &s, &c);
    float sg = a < b ? 1.0f : -1.0f;
    return V2{c * sg, s * sg};
}

// apart (fluid.wgsl:713-734)
__device__ V2 apart(const W& w, uint32_t k, uint32_t h, V2 pos, uint32_t id) {
    uint32_t start = w.gw(h, G_START), n = w.gw(h, G_SORT);
    if (n < 2u) return pos;
    const uint4* it = w.items(w.D.sorted);
    int32_t px = 0, py = 0;
    for (uint32_t m = start; m < start + n && m < w.D.cap; m++) {
        if (m == k) continue;
        uint4 o = it[m];
        float dx = pos.x - __uint_as_float(o.x), dy = pos.y - __uint_as_float(o.y);
        float l = len2(dx, dy);
        if (l < APART) {
            V2 way = l == 0.0f ? pairWay(id, it[w.D.cap + m].z) : V2{dx / l, dy / l};
            float s = 0.5f * (APART - l) * APART_FIX;
            px = (int32_t)((uint32_t)px + (uint32_t)f2i(rnd_even(s * way.x)));
            py = (int32_t)((uint32_t)py + (uint32_t)f2i(rnd_even(s * way.y)));
        }
    }
    float cx = floorf(pos.x), cy = floorf(pos.y);
    float tx = pos.x + (float)px / APART_FIX, ty = pos.y + (float)py / APART_FIX;
    V2 r;
    r.x = (tx >= cx + APART && tx <= cx + 1.0f - APART) ? tx : pos.x;
    r.y = (ty >= cy + APART && ty <= cy + 1.0f - APART) ? ty : pos.y;
    return r;
}

// rankById (fluid.wgsl:668-678)
__device__ uint32_t rankById(const W& w, uint32_t h, uint32_t k, uint32_t id, uint32_t word, uint32_t drawn) {
    uint32_t start = w.gw(h, G_START), n = w.gw(h, G_SORT);
    uint32_t mine = wordType(word) == drawn ? 1u : 0u;
    const uint4* it = w.items(w.D.sorted);
    uint32_t r = 0;
    for (uint32_t m = start; m < start + n && m < w.D.cap; m++) {
        uint4 other = it[w.D.cap + m];
        uint32_t theirs = wordType(other.x) == drawn ? 1u : 0u;
        r += (theirs < mine || (theirs == mine && (other.z < id || (other.z == id && m < k)))) ? 1u : 0u;
    }
    return r;
}

// sharedLife (fluid.wgsl:4149-4161)
__device__ uint32_t sharedLife(const W& w, uint32_t life, uint32_t was, uint32_t now, uint32_t id) {
    if (now == was) return life;
    float l = (float)life;
    if (now < was) l = l * (float)now / (float)was;
    else l = 255.0f - (255.0f - l) * (255.0f - (float)now) / (255.0f - (float)was);
    Rng g;
    g.seed(id, w.D.st->P.frame, w.D.st->P.seed ^ 0x5a17u);
    return min(f2u(floorf(l + g.next())), 255u);
}

// Warp-aggregated append to a Particles buffer's count: the first of n
// places for this thread (past capacity if there is no room).
__device__ __forceinline__ uint32_t takePlaces(uint32_t* count, uint32_t n) {
    const unsigned full = 0xffffffffu;
    unsigned lane = threadIdx.x & 31u;
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(full, incl, o);
        if (lane >= (unsigned)o) incl += v;
    }
    uint32_t total = __shfl_sync(full, incl, 31);
    uint32_t base = 0;
    if (lane == 31u && total) base = atomicAdd(count, total);
    base = __shfl_sync(full, base, 31);
    return base + incl - n;
}

__device__ __forceinline__ void storeParticle(const W& w, uint32_t m, V2 pos, V2 vel, uint32_t word, float temp, uint32_t id,
                                              float4 affine) {
    uint4* it = w.items(w.D.parts);
    it[m] = make_uint4(__float_as_uint(pos.x), __float_as_uint(pos.y), __float_as_uint(vel.x), __float_as_uint(vel.y));
    it[w.D.cap + m] = make_uint4(word, __float_as_uint(temp), id, 0u);
    it[2u * w.D.cap + m] = make_uint4(__float_as_uint(affine.x), __float_as_uint(affine.y), __float_as_uint(affine.z),
                                      __float_as_uint(affine.w));
}

// syncParticles (fluid.wgsl:767-831): a thread per particle of `sorted`.
__global__ void k_syncParticles(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
  FOR_ITEMS(Bt, L_PS, qi) {
    ITEM_WORLD_C(Bt, qi, D, w, chunk);
    uint32_t live = min(D.sorted[0], D.cap);
    uint32_t k0 = chunk * blockDim.x;
    if (k0 >= live) continue;  // whole CTA past the particles (uniform)
    uint32_t k = k0 + threadIdx.x;
    bool keep = false;
    V2 pos{0, 0}, vel{0, 0};
    uint32_t word = AIR, id = 0;
    float temp = 0.0f;
    float4 aff = make_float4(0, 0, 0, 0);
    if (k < live) {
        const uint4* it = w.items(D.sorted);
        uint4 mo = it[k], stt = it[D.cap + k], af = it[2u * D.cap + k];
        pos = V2{__uint_as_float(mo.x), __uint_as_float(mo.y)};
        vel = V2{__uint_as_float(mo.z), __uint_as_float(mo.w)};
        word = stt.x; temp = __uint_as_float(stt.y); id = stt.z;
        aff = make_float4(__uint_as_float(af.x), __uint_as_float(af.y), __uint_as_float(af.z), __uint_as_float(af.w));
        I2 hc = w.cellOf(pos.x, pos.y);
        uint32_t h = w.cellIndex(hc);
        pos = apart(w, k, h, pos, id);
        uint32_t d = w.gw(h, G_DEST);
        if (d == DEST_KEEP) {
            keep = true;
            markBlockOf(w, pos.x, pos.y);
        } else if ((d & DEST_ASIDE) != 0u && (d & ~DEST_ASIDE) < D.C) {
            uint32_t to = d & ~DEST_ASIDE;
            // not into another body's cup (fluid.wgsl:785-793)
            if (cupOf(w, to) == NONE)
                pos = V2{(float)(to % (uint32_t)D.W) + (pos.x - floorf(pos.x)), (float)(to / (uint32_t)D.W) + (pos.y - floorf(pos.y))};
            keep = true;
            markBlockOf(w, pos.x, pos.y);
        } else if (isClaim(d) && claimedCell(d) < D.C) {
            uint32_t to = claimedCell(d);
            uint4 v = w.cell(to);
            uint32_t n = liquidCount(v.w);
            if (n == LIQUID_COUNT_MAX || w.gw(h, G_SORT) <= n || rankById(w, h, k, id, word, wordType(v.x)) < n) {
                if (to != h)
                    pos = V2{(float)(to % (uint32_t)D.W) + (pos.x - floorf(pos.x)), (float)(to / (uint32_t)D.W) + (pos.y - floorf(pos.y))};
                temp = __uint_as_float(v.y);
                uint32_t drawn = w.gw(h, G_TYPE);
                uint32_t pt = wordType(word);
                if (holdsSolute(pt) && pt == (drawn & 0xffu) && wordType(v.x) == pt &&
                    (wordAux(word) == ((drawn >> 8u) & 0xffu) || wordAux(word) == 0u)) {
                    uint32_t life = sharedLife(w, wordAux(word) == 0u ? 0u : wordLife(word), (drawn >> 16u) & 0xffu, wordLife(v.x), id);
                    uint32_t ww = wordWithout(v.x, FL_DRAWN);
                    uint32_t solute = wordAux(ww) != 0u ? wordAux(ww) : ((drawn >> 8u) & 0xffu);
                    word = packWord(pt, life > 0u ? solute : 0u, life, wordShade(ww), wordFlags(ww));
                } else if (drawnAs(word) == (drawn & 0xffffu)) {
                    word = wordWithout(v.x, FL_DRAWN);
                }
                keep = true;
            }
        }
    }
    uint32_t m = takePlaces(&D.parts[0], keep ? 1u : 0u);
    if (keep && m < D.cap) storeParticle(w, m, pos, vel, word, temp, id, aff);
  }
}

// seedId, seedPos (fluid.wgsl:835-855)
__device__ uint32_t seedId(const Dev& D, I2 c, uint32_t j) {
    uint32_t h = (((uint32_t)c.y * (uint32_t)D.W + (uint32_t)c.x) * 0x9e3779b9u) ^ (D.st->P.frame * 0x85ebca6bu) ^ (j * 0xc2b2ae35u);
    h ^= h >> 16u;
    h *= 0x7feb352du;
    h ^= h >> 15u;
    return h;
}

// syncSeed (fluid.wgsl:863-890): a CTA per block of the world.
__global__ void k_syncSeed(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
  FOR_ITEMS(Bt, L_WB, qi) {
    ITEM_WORLD_C(Bt, qi, D, w, blk);
    if (D.st->book) continue;
    const I2 bq_ = w.blockAt(blk);
    I2 c{bq_.x * BLOCK + (int)(threadIdx.x & 7u), bq_.y * BLOCK + (int)(threadIdx.x >> 3)};
    uint32_t n = 0;
    uint4 v = make_uint4(0, 0, 0, 0);
    Rng g;
    g.s = 0;
    if (w.inWorld(c)) {
        uint32_t i = w.cellIndex(c);
        v = w.cell(i);
        if (w.kindOf(wordType(v.x)) == WIG_KIND_LIQUID) {
            uint32_t home = liquidHome(v.w);
            uint32_t want = liquidCount(v.w);
            if (!wordHas(v.x, FL_DRAWN)) n = D.ppc;
            else if (home >= D.C || w.gw(home, G_DEST) != claimOf(i)) n = max(want, 1u);
            else if (want > w.gw(home, G_SORT) && want < LIQUID_COUNT_MAX) n = want - w.gw(home, G_SORT);
            g.seed(i, D.st->P.frame, D.st->P.seed ^ 0x5eedu);
        }
    }
    uint32_t m = takePlaces(&D.parts[0], n);
    for (uint32_t j = 0; j < n; j++) {
        V2 pos;
        if (n == 1u) {
            pos = V2{(float)c.x + 0.5f, (float)c.y + 0.5f};
        } else {
            float rx = g.next();
            float ry = g.next();
            float r0 = rx - 0.5f, r1 = ry - 0.5f;
            if (n <= 4u) {
                float qx = (j == 1u || j == 2u) ? 1.0f : 0.0f, qy = (j == 1u || j == 3u) ? 1.0f : 0.0f;
                pos = V2{(float)c.x + 0.25f + 0.5f * qx + 0.3f * r0, (float)c.y + 0.25f + 0.5f * qy + 0.3f * r1};
            } else {
                pos = V2{(float)c.x + 0.5f + 0.9f * r0, (float)c.y + 0.5f + 0.9f * r1};
            }
        }
        if (m + j < D.cap) {
            V2 vel{f16_value(v.z & 0xffffu), f16_value(v.z >> 16)};
            storeParticle(w, m + j, pos, vel, wordWithout(v.x, FL_DRAWN), __uint_as_float(v.y), seedId(D, c, j),
                          make_float4(0, 0, 0, 0));
        }
    }
  }
}

// The marks of block b's 3x3 neighbourhood (OR of the blocks inside the world).
__device__ __forceinline__ uint32_t marksAround(const W& w, I2 b) {
    uint32_t m[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const I2 o{b.x + k % 3 - 1, b.y + k / 3 - 1};
        m[k] = w.inBlocks(o) ? w.D.blocks[w.blockIndex(o)] : 0u;
    }
    uint32_t marks = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) marks |= m[k];
    return marks;
}

// compact (fluid.wgsl:896-921): one 1024-thread CTA a world, each thread a
// run of consecutive blocks, so the lists come out in block-index order.  The first pass reads every block's marks and
// state (four blocks' loads issued together) and keeps what it found, a bit
// a block, for the second (runs of up to 64 blocks; a longer run reads them
// again), which writes the states and the lists in block order after the
// scan of the runs' counts.
__global__ void __launch_bounds__(1024) k_compact(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    __shared__ uint32_t sa[1024], sr[1024];
    FOR_ITEMS(Bt, L_ONE_ALL, it) {
        ITEM_WORLD_C(Bt, it, D, w, unused_);
        (void)unused_;
        const uint32_t per = (D.B + 1023u) / 1024u;
        const uint32_t lo = min(threadIdx.x * per, D.B), hi = min(lo + per, D.B);
        const bool keep = per <= 64u;
        uint64_t liq = 0, nea = 0, wasm = 0;
        uint32_t na = 0, nr = 0;
#pragma unroll 4
        for (uint32_t n = lo; n < hi; n++) {
            const uint32_t marks = marksAround(w, w.blockAt(n));
            const bool liquid = (marks & (MARK_LIQUID | MARK_REGION)) != 0u;
            const bool was = (D.blocks[w.stateSlot(n)] & ACTIVE) != 0u;
            const uint64_t bit = 1ull << ((n - lo) & 63u);
            if (liquid) liq |= bit;
            if ((marks & MARK_LIQUID) != 0u) nea |= bit;
            if (was) wasm |= bit;
            na += liquid ? 1u : 0u;
            nr += (!liquid && was) ? 1u : 0u;
        }
        sa[threadIdx.x] = na;
        sr[threadIdx.x] = nr;
        __syncthreads();
        for (uint32_t o = 1; o < 1024u; o <<= 1) {
            uint32_t a = threadIdx.x >= o ? sa[threadIdx.x - o] : 0u;
            uint32_t r = threadIdx.x >= o ? sr[threadIdx.x - o] : 0u;
            __syncthreads();
            sa[threadIdx.x] += a;
            sr[threadIdx.x] += r;
            __syncthreads();
        }
        uint32_t ai = sa[threadIdx.x] - na, ri = sr[threadIdx.x] - nr;
        // All states are read above before any is written below.
        __syncthreads();
        for (uint32_t n = lo; n < hi; n++) {
            bool liquid, near, was;
            if (keep) {
                const uint64_t bit = 1ull << (n - lo);
                liquid = (liq & bit) != 0u;
                near = (nea & bit) != 0u;
                was = (wasm & bit) != 0u;
            } else {
                const uint32_t marks = marksAround(w, w.blockAt(n));
                liquid = (marks & (MARK_LIQUID | MARK_REGION)) != 0u;
                near = (marks & MARK_LIQUID) != 0u;
                was = (D.blocks[w.stateSlot(n)] & ACTIVE) != 0u;
            }
            D.blocks[w.stateSlot(n)] = (liquid ? ACTIVE : 0u) | (near ? NEAR_LIQUID : 0u);
            if (liquid) D.blocks[w.activeSlot(ai++)] = n;
            else if (was) D.blocks[w.retiredSlot(ri++)] = n;
        }
        if (threadIdx.x == 1023u) {
            D.blocks[w.countSlot(COUNT_ACTIVE)] = sa[1023];
            D.blocks[w.countSlot(COUNT_RETIRED)] = sr[1023];
        }
        __syncthreads();
    }
}

// retire (fluid.wgsl:924-951)
__global__ void k_retire(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_RET, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        uint32_t n = D.blocks[w.retiredSlot(wid)];
        const I2 bq_ = w.blockAt(n);
        I2 c{bq_.x * BLOCK + (int)(threadIdx.x & 7u), bq_.y * BLOCK + (int)(threadIdx.x >> 3)};
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        reinterpret_cast<float4*>(D.field)[2u * i] = make_float4(0, 0, 0, 0);
        reinterpret_cast<float4*>(D.field)[2u * i + 1u] = make_float4(0, 0, 0, 0);
        for (uint32_t g = 0; g < CELL_WORDS; g++) *w.gwp(i, g) = 0u;
        int fs[4][3];
        w.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            uint32_t f = w.faceIndex(I2{fs[j][0], fs[j][1]}, fs[j][2] == 1);
            reinterpret_cast<float4*>(D.field)[w.faceSlot(f)] = make_float4(0, 0, 0, 0);
            *w.viscLastP(f) = 0.0f;
            D.counters[w.sumSlot(f)] = 0u;
            D.counters[w.sumSlot(f) + 1u] = 0u;
        }
        if (threadIdx.x == 0) D.blocks[n] = 0u;
    }
}

// clear (fluid.wgsl:962-985)
__global__ void k_clear(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 b = w.activeBlock(wid);
        if (threadIdx.x == 0) D.blocks[w.blockIndex(b)] = 0u;
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        for (uint32_t g = 0; g < CELL_WORDS; g++) *w.gwp(i, g) = 0u;
        *w.gwp(i, G_REGION) = i;
        int fs[4][3];
        w.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            uint32_t f = w.faceIndex(I2{fs[j][0], fs[j][1]}, fs[j][2] == 1);
            D.counters[w.sumSlot(f)] = 0u;
            D.counters[w.sumSlot(f) + 1u] = 0u;
        }
    }
}

// ================================================================ splat

// splatAxis (fluid.wgsl:1000-1015)
// Where the splat's fixed-point adds go.  DirectSink: global atomics, a site
// at a time.  WinSink: a warp's window in shared memory, summed there and
// added to the global words once a site (WarpGather); the sums are
// integers, so the words end as with every add made alone.
struct DirectSink {
    const W& w;
    __device__ __forceinline__ void face(bool isU, I2 at, uint32_t a, uint32_t b) const {
        uint32_t slot = w.sumSlot(w.faceIndex(at, isU));
        atomicAdd(&w.D.counters[slot], a);
        atomicAdd(&w.D.counters[slot + 1u], b);
    }
    __device__ __forceinline__ void cell(uint32_t g, I2 at, uint32_t v) const { atomicAdd(w.gwp(w.cellIndex(at), g), v); }
};

// A warp's window: the sites of (GWX + 1) x (GWY + 1) coordinates from
// (x0, y0): per u face and v face its two sums, per cell its count, mass
// and density words.
constexpr int GWX = 16, GWY = 8, GWN = (GWX + 1) * (GWY + 1);
struct GatherWin {
    uint32_t u[2][GWN], v[2][GWN], c[3][GWN];
};
struct WinSink {
    GatherWin& win;
    int x0, y0;
    __device__ __forceinline__ int at_(I2 at) const { return (at.y - y0) * (GWX + 1) + (at.x - x0); }
    __device__ __forceinline__ void face(bool isU, I2 at, uint32_t a, uint32_t b) const {
        const int e = at_(at);
        uint32_t(*arr)[GWN] = isU ? win.u : win.v;
        atomicAdd(&arr[0][e], a);
        atomicAdd(&arr[1][e], b);
    }
    __device__ __forceinline__ void cell(uint32_t g, I2 at, uint32_t v) const {
        atomicAdd(&win.c[g == G_COUNT ? 0 : g == G_MASS ? 1 : 2][at_(at)], v);
    }
};

// splatAxis (fluid.wgsl:1041-1067): a face's fixed-point sums of v w and w.
template <class Sink>
__device__ __forceinline__ void splatAxis(const W& w, const Sink& k, float sx, float sy, float vel, float gx, float gy,
                                          bool isU) {
    float fx0 = floorf(sx), fy0 = floorf(sy);
    int bx = f2i(fx0), by = f2i(fy0);
    float fx = sx - fx0, fy = sy - fy0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int ox = j & 1, oy = j >> 1;
        float wgt = (ox == 1 ? fx : 1.0f - fx) * (oy == 1 ? fy : 1.0f - fy);
        I2 at{bx + ox, by + oy};
        if (wgt <= 0.0f || !w.faceInWorld(at, isU)) continue;
        float there = vel + (gx * ((float)at.x - sx) + gy * ((float)at.y - sy));
        k.face(isU, at, (uint32_t)f2i(rnd_even(there * wgt * FIX)), (uint32_t)f2i(rnd_even(wgt * FIX)));
    }
}
__device__ __forceinline__ bool walls(const W& w, I2 c) {
    if (!w.inWorld(c)) return true;
    uint32_t k = w.kindOfCell(w.cellIndex(c));
    return k == WIG_KIND_SOLID || k == WIG_KIND_POWDER;
}
// splatDensity (fluid.wgsl:1069-1087)
template <class Sink>
__device__ __forceinline__ void splatDensity(const W& w, const Sink& k, float px, float py, float room) {
    float sx = px - 0.5f, sy = py - 0.5f;
    float fx0 = floorf(sx), fy0 = floorf(sy);
    int bx = f2i(fx0), by = f2i(fy0);
    float fx = sx - fx0, fy = sy - fy0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int ox = j & 1, oy = j >> 1;
        float wgt = (ox == 1 ? fx : 1.0f - fx) * (oy == 1 ? fy : 1.0f - fy);
        I2 at{bx + ox, by + oy};
        if (walls(w, at)) {
            I2 x{bx + 1 - ox, at.y}, y{at.x, by + 1 - oy}, xy{bx + 1 - ox, by + 1 - oy};
            if (!walls(w, x)) at = x;
            else if (!walls(w, y)) at = y;
            else if (!walls(w, xy)) at = xy;
            else at = I2{-1, -1};
        }
        if (w.inWorld(at) && wgt > 0.0f) k.cell(G_DENSITY, at, f2u(rnd_even(wgt * room * FIX)));
    }
}

// gather (fluid.wgsl:1017-1039) of one particle, no air bound: no air push.
struct GatherIn {
    float px, py, vx, vy, temp;
    uint4 stt, af;
};
template <class Sink>
__device__ __forceinline__ void gatherTo(const W& w, const Sink& k, const GatherIn& p) {
    splatAxis(w, k, p.px - 0.0f, p.py - 0.5f, p.vx, __uint_as_float(p.af.x), __uint_as_float(p.af.y), true);
    splatAxis(w, k, p.px - 0.5f, p.py - 0.0f, p.vy, __uint_as_float(p.af.z), __uint_as_float(p.af.w), false);
    const I2 home = w.cellOf(p.px, p.py);
    k.cell(G_COUNT, home, 1u);
    k.cell(G_MASS, home, f2u(rnd_even(w.liquidDensity(p.stt.x, p.temp) * FIX)));
    splatDensity(w, k, p.px, p.py, w.liquidVolume(p.stt.x, p.temp));
}

// A warp's 32 particles of `parts` (in cell order, so mostly a few
// neighbouring cells): when every site they add to fits one window, summed
// there and flushed once a site; else each particle's adds straight to the
// global words.
__device__ __forceinline__ void gatherWarp(const Dev& D, const W& w, uint32_t k, GatherWin& win) {
    const uint32_t live = min(D.parts[0], D.cap);
    const bool has = k < live;
    GatherIn p{};
    int lx = 0x3fffffff, ly = 0x3fffffff, hx = -0x3fffffff, hy = -0x3fffffff;
    if (has) {
        const uint4* it = w.items(D.parts);
        const uint4 mo = it[k];
        p.stt = it[D.cap + k];
        p.af = it[2u * D.cap + k];
        p.px = __uint_as_float(mo.x);
        p.py = __uint_as_float(mo.y);
        p.vx = __uint_as_float(mo.z);
        p.vy = __uint_as_float(mo.w);
        p.temp = __uint_as_float(p.stt.y);
        // the sites' coordinates: x from floor(px - 1/2) to floor(px) + 1,
        // y likewise, and the (clamped) home cell; a position far outside
        // any world (or not a number) sends the warp the direct way
        if (fabsf(p.px) < 1.0e6f && fabsf(p.py) < 1.0e6f) {
            const I2 home = w.cellOf(p.px, p.py);
            lx = min(f2i(floorf(p.px - 0.5f)), home.x);
            ly = min(f2i(floorf(p.py - 0.5f)), home.y);
            hx = max(f2i(floorf(p.px)) + 1, home.x);
            hy = max(f2i(floorf(p.py)) + 1, home.y);
        } else {
            lx = ly = -0x3fffffff;
            hx = hy = 0x3fffffff;
        }
    }
    const int x0 = __reduce_min_sync(0xffffffffu, lx), y0 = __reduce_min_sync(0xffffffffu, ly);
    const int x1 = __reduce_max_sync(0xffffffffu, hx), y1 = __reduce_max_sync(0xffffffffu, hy);
    if (x1 - x0 > GWX || y1 - y0 > GWY) {  // (warp-uniform)
        if (has) gatherTo(w, DirectSink{w}, p);
        return;
    }
    if (x1 < x0) return;  // no particle in the warp
    if (has) gatherTo(w, WinSink{win, x0, y0}, p);
    __syncwarp();
    // the flush: the sites' box alone (every add fell inside it), a lane a
    // window entry; each nonzero sum added to its global word and cleared
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t bw = (uint32_t)(x1 - x0 + 1), nbox = bw * (uint32_t)(y1 - y0 + 1);
    for (uint32_t q = lane; q < nbox; q += 32u) {
        const uint32_t qy = q / bw, qx = q - qy * bw;
        const uint32_t e = qy * (uint32_t)(GWX + 1) + qx;
        const I2 at{x0 + (int)qx, y0 + (int)qy};
        for (int isU = 1; isU >= 0; isU--) {
            uint32_t(*arr)[GWN] = isU ? win.u : win.v;
            const uint32_t a = arr[0][e], b = arr[1][e];
            if ((a | b) == 0u) continue;
            arr[0][e] = 0u;
            arr[1][e] = 0u;
            const uint32_t slot = w.sumSlot(w.faceIndex(at, isU != 0));
            atomicAdd(&D.counters[slot], a);
            atomicAdd(&D.counters[slot + 1u], b);
        }
        const uint32_t g3[3] = {G_COUNT, G_MASS, G_DENSITY};
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const uint32_t v = win.c[j][e];
            if (v == 0u) continue;
            win.c[j][e] = 0u;
            atomicAdd(w.gwp(w.cellIndex(at), g3[j]), v);
        }
    }
    __syncwarp();
}
__global__ void __launch_bounds__(256) k_gather(Batch Bt) {
    __shared__ WorldCopy wc_;
    __shared__ GatherWin win_[8];
    worldCopyInit(wc_);
    GatherWin& win = win_[threadIdx.x >> 5];
    {
        uint32_t* z = &win.u[0][0];
        for (uint32_t i = threadIdx.x & 31u; i < sizeof(GatherWin) / 4u; i += 32u) z[i] = 0u;
        __syncwarp();
    }
    FOR_ITEMS(Bt, L_PP, qi) {
        ITEM_WORLD_C(Bt, qi, D, w, chunk);
        gatherWarp(D, w, chunk * blockDim.x + threadIdx.x, win);
    }
}

// ================================================================ classify

__device__ bool mayBeSealed(const W& w, I2 c) {
    if (countAt(w, c) != 0) return false;
    uint32_t i = w.cellIndex(c);
    return w.fv(2u * i)[2] > 0.0f || w.fv(2u * i + 1u)[2] != 0.0f;
}
__device__ bool wasOpen(const W& w, I2 q) {
    if (!w.inWorld(q) || countAt(w, q) < 0) return false;
    uint32_t sb = 1u << ((w.D.st->P.frame + 1u) & 1u);
    return (f2u(w.fv(2u * w.cellIndex(q) + 1u)[3]) & sb) == 0u;
}

// sealJoin (fluid.wgsl:1531-1543)
__global__ void k_sealJoin(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c) || !mayBeSealed(w, c)) continue;
        for (int d = 0; d < 2; d++) {
            I2 n = d == 0 ? I2{c.x + 1, c.y} : I2{c.x, c.y + 1};
            if (mayBeSealed(w, n)) ufJoin(w, w.cellIndex(c), w.cellIndex(n));
        }
    }
}
// sealAnchor (fluid.wgsl:1545-1554)
__global__ void k_sealAnchor(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c) || !mayBeSealed(w, c)) continue;
        if (wasOpen(w, beside(c, 0)) || wasOpen(w, beside(c, 1)) || wasOpen(w, beside(c, 2)) || wasOpen(w, beside(c, 3)))
            atomicOr(w.gwp(ufFind(w, w.cellIndex(c)), G_REGION), REGION_OPEN);
    }
}

// columnWeight (fluid.wgsl:1566-1575): the cells with particles straight
// above p, counted up to the first without (at most COLUMN_MOST).  The
// column is read COLUMN_RUN cells at a time, their type and count words
// loaded together; each cell's countAt then follows from those words (the
// full test only for a gas cell, which may be a bubble), and the cells are
// taken in order, as the walk takes them.
constexpr int COLUMN_RUN = 8;
__device__ float columnWeight(const W& w, I2 p, float density) {
    int over = 0;
    int y = p.y - 1;
    bool more = true;
    while (more && over < COLUMN_MOST) {
        uint32_t t[COLUMN_RUN], n[COLUMN_RUN];
        bool in[COLUMN_RUN];
#pragma unroll
        for (int k = 0; k < COLUMN_RUN; k++) {
            const I2 q{p.x, y - k};
            in[k] = w.inWorld(q);
            const uint32_t i = in[k] ? w.cellIndex(q) : 0u;
            t[k] = w.cellType(i);
            n[k] = w.gw(i, G_COUNT);
        }
#pragma unroll
        for (int k = 0; k < COLUMN_RUN; k++) {
            int m = -1;
            if (in[k]) {
                const uint32_t kind = w.kindOf(t[k]);
                if (kind == WIG_KIND_GAS) m = countAt(w, I2{p.x, y - k});
                else if (kind != WIG_KIND_SOLID && kind != WIG_KIND_POWDER) m = (int32_t)n[k];
            }
            if (more && over < COLUMN_MOST && m > 0) over += 1;
            else more = false;
        }
        y -= COLUMN_RUN;
    }
    return density * w.D.st->P.earth_g * ((float)over + 0.5f);
}

// classify (fluid.wgsl:1578-1696), no bodies.
__global__ void k_classify(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    __shared__ uint32_t blockBits;
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        const uint32_t frame = D.st->P.frame;
        const uint32_t mine = 1u << (frame & 1u), fall0 = 4u << (frame & 1u);
        if (threadIdx.x == 0) blockBits = 0u;
        __syncthreads();
        I2 p = lidCell(w, wid);
        if (w.inWorld(p)) {
            uint32_t i = w.cellIndex(p);
            int n = countAt(w, p);
            float4 c = make_float4(0, 0, 0, 0);
            float4 was = w.f4(2u * i), wasDrift = w.f4(2u * i + 1u);
            bool sealed = false;
            if (n == 0 && mayBeSealed(w, p)) sealed = (vload(w.gwp(ufFind(w, i), G_REGION)) & REGION_OPEN) == 0u;
            uint32_t rigid = NONE, held = NONE;
            const uint32_t seam = n < 0 ? NONE : seamOf(w, i);
            if (seam != NONE) {
                // a gap the stamp opened in a body's wall: the body's (fluid.wgsl:1604-1613)
                c.z = -1.0f;
                rigid = seam;
                if (isHeld(w, seam)) {
                    held = seam;
                    rigid = NONE;
                }
                sealed = false;
            } else if (n < 0) {
                c.z = -1.0f;
                // a free body's cell, or powder in its cup, its cargo (fluid.wgsl:1614-1627)
                if (D.motion) {
                    rigid = rigidBodyOf(w, w.cell(i));
                    if (rigid == NONE && w.kindOfCell(i) == WIG_KIND_POWDER) rigid = cupOf(w, i);
                }
                if (rigid != NONE && isHeld(w, rigid)) {
                    held = rigid;
                    rigid = NONE;
                }
            } else if (n > 0) {
                V2 li = liquidIn(w, i);
                c = make_float4(0.0f, 0.0f, li.x, li.y);
            } else {
                float fluid = 0.0f, wallsN = 0.0f;
                V2 mean{0.0f, 0.0f};
                for (int d = 0; d < 4; d++) {
                    I2 q = beside(p, d);
                    int m = countAt(w, q);
                    if (m < 0) wallsN = wallsN + 1.0f;
                    else if (m > 0) {
                        fluid = fluid + 1.0f;
                        V2 li = liquidIn(w, w.cellIndex(q));
                        mean.x = mean.x + li.x;
                        mean.y = mean.y + li.y;
                    }
                }
                if (fluid >= 2.0f && fluid + wallsN >= 3.0f) c = make_float4(0.0f, 0.0f, mean.x / fluid, mean.y / fluid);
                else if (sealed) c = fluid > 0.0f ? make_float4(0.0f, 0.0f, mean.x / fluid, mean.y / fluid) : make_float4(0.0f, 0.0f, 1.0f, 0.0f);
            }
            uint32_t liquid = (c.z > 0.0f || rigid != NONE || held != NONE) ? mine : 0u;
            float4 drift = make_float4(0.0f, 0.0f, sealed ? 1.0f : 0.0f, (float)((f2u(wasDrift.w) & ~(mine | fall0)) | liquid));
            if (rigid != NONE) drift.z = -1.0f - (float)rigid;
            else if (held != NONE) drift.z = -1.0f - (float)(held + MAX_BODIES);
            if (c.z > 0.0f) {
                if (was.z > 0.0f) {
                    c.x = was.x;
                    drift.x = wasDrift.x * DRIFT_KEEP;
                } else {
                    c.x = columnWeight(w, p, c.z);
                }
                atomicOr(&blockBits, c.w > 0.0f ? (HAS_FLUID | HAS_VISCOUS) : HAS_FLUID);
            }
            reinterpret_cast<float4*>(D.field)[2u * i] = c;
            reinterpret_cast<float4*>(D.field)[2u * i + 1u] = drift;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t bits = blockBits;
            atomicOr(&D.blocks[w.stateSlot(w.blockIndex(w.activeBlock(wid)))], bits);
            if (bits & HAS_VISCOUS) D.blocks[w.countSlot(COUNT_VISCOUS)] = 1u;
        }
        __syncthreads();
    }
}

// ================================================================ faces

__device__ float obstacleVelAxis(const W& w, I2 c, int axis) {
    if (!w.inWorld(c)) return 0.0f;
    uint4 v = w.cell(w.cellIndex(c));
    uint32_t k = w.kindOf(wordType(v.x));
    if (k == WIG_KIND_SOLID || k == WIG_KIND_GAS) return 0.0f;
    float cv = axis == 0 ? f16_value(v.z & 0xffffu) : f16_value(v.z >> 16);
    return cv * POWDER_PUSH;
}
__device__ float faceViscosity(float4 ga, float4 gb) {
    if (ga.z < 0.0f || gb.z < 0.0f) return 0.0f;
    float fa = ga.z > 0.0f ? 1.0f : 0.0f, fb = gb.z > 0.0f ? 1.0f : 0.0f;
    return (fa * ga.w + fb * gb.w) / fmaxf(fa + fb, 1.0f);
}
__device__ bool wasLiquid(const W& w, I2 c) {
    uint32_t sb = 1u << ((w.D.st->P.frame + 1u) & 1u);
    return (f2u(w.fv(2u * w.cellIndex(c) + 1u)[3]) & sb) != 0u;
}
__device__ float lastPush(const W& w, I2 a, I2 at, float4 ga, float4 gb) {
    if ((ga.z > 0.0f && !wasLiquid(w, a)) || (gb.z > 0.0f && !wasLiquid(w, at))) return 0.0f;
    return fineBeta(ga.z, gb.z, w.densityAt(a), w.densityAt(at)) * (gb.x - ga.x);
}

// setBodyFace (fluid.wgsl:1840-1859)
__device__ void setBodyFace(const W& w, uint32_t f, I2 at, bool isU, float4 ga, float4 gb, uint32_t ra, uint32_t rb,
                            bool drag) {
    const V2 x = faceMiddle(at, isU);
    float now = 0.0f, u = 0.0f;
    if (ra != NONE && rb != NONE) {
        const V2 ma = bodyMoving(w, ra, x, drag), mb = bodyMoving(w, rb, x, drag);
        const V2 va = rigidVel(w, ra, x), vb = rigidVel(w, rb, x);
        now = 0.5f * (isU ? ma.x + mb.x : ma.y + mb.y);
        u = 0.5f * (isU ? va.x + vb.x : va.y + vb.y);
    } else {
        const uint32_t b = ra != NONE ? ra : rb;
        const V2 m = bodyMoving(w, b, x, drag), v = rigidVel(w, b, x);
        now = isU ? m.x : m.y;
        u = isU ? v.x : v.y;
    }
    const float4 other = ra != NONE ? gb : ga;
    const float nu = ((ra == NONE || rb == NONE) && other.z > 0.0f) ? other.w : 0.0f;
    reinterpret_cast<float4*>(w.D.field)[w.faceSlot(f)] = make_float4(now, u, 1.0f, nu);
    *w.viscRhsP(f) = now;
}

// setFace (fluid.wgsl:1936-1980), no air bound: no wind drag.
__device__ void setFace(const W& w, I2 at, bool isU) {
    uint32_t f = w.faceIndex(at, isU);
    I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
    int axis = isU ? 0 : 1;
    float4 ga = w.gridAt(a), gb = w.gridAt(at);
    if (w.D.motion) {
        const uint32_t ra = rigidAt(w, a), rb = rigidAt(w, at);
        if (ra != NONE || rb != NONE) {
            setBodyFace(w, f, at, isU, ga, gb, ra, rb, false);
            return;
        }
    }
    uint32_t slot = w.sumSlot(f);
    int32_t weight = (int32_t)w.D.counters[slot + 1u];
    float u = 0.0f, held = 0.0f;
    if (ga.z < 0.0f && gb.z < 0.0f) {
        held = -1.0f;
    } else if (ga.z < 0.0f || gb.z < 0.0f) {
        u = obstacleVelAxis(w, ga.z < 0.0f ? a : at, axis);
        held = 1.0f;
    } else if (weight > 0) {
        u = (float)(int32_t)w.D.counters[slot] / (float)weight;
        held = 1.0f;
    }
    float now = u;
    if (held > 0.0f && ga.z >= 0.0f && gb.z >= 0.0f) {
        V2 pl = w.pull();
        now = now + (isU ? pl.x : pl.y);
    }
    float start = now;
    float fvisc = faceViscosity(ga, gb);
    if (fvisc > 0.0f) {
        now = now - lastPush(w, a, at, ga, gb);
        start = now + *w.viscLastP(f);
    }
    reinterpret_cast<float4*>(w.D.field)[w.faceSlot(f)] = make_float4(start, u, held, fvisc);
    *w.viscRhsP(f) = now;
}

// setFaces (fluid.wgsl:1982-1994)
__global__ void k_setFaces(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        int fs[4][3];
        w.facesOf(c, fs);
        for (int j = 0; j < 4; j++)
            if (fs[j][2] >= 0) setFace(w, I2{fs[j][0], fs[j][1]}, fs[j][2] == 1);
    }
}

// viscousFace (fluid.wgsl:3347-3403)
__device__ void viscousFace(const W& w, I2 at, bool isU, int color) {
    if (((at.x + at.y) & 1) != color) return;
    I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
    float4 ga = w.gridAt(a), gb = w.gridAt(at);
    const uint32_t ra = rigidAt(w, a), rb = rigidAt(w, at);
    const bool surface = (ra != NONE) != (rb != NONE) && (ra != NONE ? gb.z : ga.z) > 0.0f;
    if (!surface && (ga.z < 0.0f || gb.z < 0.0f || ra != NONE || rb != NONE)) return;
    uint32_t fi = w.faceIndex(at, isU);
    float* fp = w.fv(w.faceSlot(fi));
    float nu = fp[3];
    if (nu <= 0.0f) return;
    float heavy = 1.0f;
    if (surface) {
        const float liquid = ra != NONE ? gb.z : ga.z;
        heavy = 2.0f * liquid / (liquid + bodyDensity(w, ra != NONE ? ra : rb));
    }
    float tx = ga.z > 0.0f ? ga.w : 0.0f, ty = gb.z > 0.0f ? gb.w : 0.0f;
    float sum = 0.0f, n = 0.0f;
    for (int d = 0; d < 4; d++) {
        I2 o = beside(at, d);
        bool across = isU == (d >= 2);
        float4 other = make_float4(0.0f, 0.0f, -1.0f, 0.0f);
        if (w.faceInWorld(o, isU)) other = w.f4(w.faceSlot(w.faceIndex(o, isU)));
        float k = (d & 1) == 1 ? ty : tx;
        if (across) k = other.z < 0.0f ? nu : 2.0f * nu * other.w / fmaxf(nu + other.w, 1e-12f);
        if (other.z < 0.0f) n = n + k * (across ? 2.0f : 1.0f);
        else if (other.z > 0.0f) { sum = sum + k * other.x; n = n + k; }
    }
    fp[0] = mixf(fp[0], (*w.viscRhsP(fi) + heavy * sum) / (1.0f + heavy * n), VISC_OMEGA);
}

// viscosityRed / viscosityBlack / unpress (fluid.wgsl:3409-3466)
__global__ void k_viscosity(Batch Bt, int color) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        if (color < 2 && D.st->viscous == 0u) continue;  // this world's step has no sweeps
        I2 b = w.activeBlock(wid);
        if ((w.statesOf(I2{b.x - 1, b.y - 1}, I2{b.x + 1, b.y + 1}) & HAS_VISCOUS) == 0u) continue;
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        int fs[4][3];
        w.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            I2 at{fs[j][0], fs[j][1]};
            bool isU = fs[j][2] == 1;
            if (color < 2) {
                viscousFace(w, at, isU, color);
                continue;
            }
            I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
            float4 ga = w.gridAt(a), gb = w.gridAt(at);
            uint32_t fi = w.faceIndex(at, isU);
            if (rigidAt(w, a) == NONE && rigidAt(w, at) == NONE && faceViscosity(ga, gb) > 0.0f) {
                float* fp = w.fv(w.faceSlot(fi));
                *w.viscLastP(fi) = fp[0] - *w.viscRhsP(fi);
                fp[0] = fp[0] + lastPush(w, a, at, ga, gb);
            } else if (*w.viscLastP(fi) != 0.0f) {
                *w.viscLastP(fi) = 0.0f;
            }
        }
    }
}

// divergence (fluid.wgsl:1996-2025)
__global__ void k_divergence(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    // once a world: its residual and iteration words cleared
    if (threadIdx.x == 0) {
        FOR_ITEMS(Bt, L_ONE, ot) {
            ITEM_WORLD(Bt, ot, D, w, unused_);
            (void)unused_;
            D.blocks[w.countSlot(COUNT_RESIDUAL)] = 0u;
            D.blocks[w.countSlot(COUNT_CYCLES)] = 0u;
        }
    }
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        if (w.fv(2u * i)[2] <= 0.0f) continue;
        float out = w.fv(w.faceSlot(w.uFace(c.x + 1, c.y)))[0] - w.fv(w.faceSlot(w.uFace(c.x, c.y)))[0] +
                    w.fv(w.faceSlot(w.vFace(c.x, c.y + 1)))[0] - w.fv(w.faceSlot(w.vFace(c.x, c.y)))[0];
        w.fv(2u * i)[1] = out;
        float n = w.densityAt(c);
        float room = posedRoom(w, c);
        w.fv(2u * i + 1u)[1] = w.fv(2u * i + 1u)[2] < 0.0f ? 0.0f : -SPREAD * (n - room);
    }
}

// ================================================================ the solve's start

// cgStart (fluid.wgsl:2665-2674)
__global__ void k_cgStart(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        reinterpret_cast<float4*>(D.cg)[i] = make_float4(w.gridAt(c).x, 0.0f, 0.0f, 0.0f);
        *w.gwp(i, G_REGION) = i;
    }
}
// cgJoin (fluid.wgsl:2677-2689)
__global__ void k_cgJoin(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c) || w.gridAt(c).z <= 0.0f) continue;
        for (int d = 0; d < 2; d++) {
            I2 n = d == 0 ? I2{c.x + 1, c.y} : I2{c.x, c.y + 1};
            if (rhoAt(w, 0, n) > 0.0f) ufJoin(w, w.cellIndex(c), w.cellIndex(n));
        }
    }
}
// cgStart with the block's own part of cgJoin's labelling, for the fast
// forms' steps (the per-pass dispatch and the plain form keep k_cgStart and
// k_cgJoin): each liquid cell's region link goes straight to the smallest
// index of the liquid cells its block joins it to (min-label propagation
// over the block's 4-neighbour liquid edges in shared memory, at most 63
// rounds), every other cell its own root.  The union-find's links always
// point to lower indices and its roots are the smallest indices of their
// regions, so after k_cgJoinAcross has joined the edges between blocks the
// regions, their roots and every ufFind are those of cgJoin's; only the
// intermediate links, a lock-free union-find's timing in the reference too,
// differ (cgFinish clears them all).
__global__ void k_cgStartLocal(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    __shared__ uint32_t lab[64];
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        const I2 c = lidCell(w, wid);
        const bool in = w.inWorld(c);
        const uint32_t i = in ? w.cellIndex(c) : 0u;
        bool fluid = false;
        if (in) {
            const float4 g = w.gridAt(c);
            reinterpret_cast<float4*>(D.cg)[i] = make_float4(g.x, 0.0f, 0.0f, 0.0f);
            fluid = g.z > 0.0f;
        }
        const int t = (int)threadIdx.x, lx = t & 7, ly = t >> 3;
        lab[t] = fluid ? i : 0xffffffffu;
        __syncthreads();
        for (int round = 0; round < 64; round++) {
            uint32_t m = lab[t];
            if (fluid) {
                if (lx > 0) m = min(m, lab[t - 1]);
                if (lx < 7) m = min(m, lab[t + 1]);
                if (ly > 0) m = min(m, lab[t - 8]);
                if (ly < 7) m = min(m, lab[t + 8]);
            }
            __syncthreads();
            const bool changed = m < lab[t];
            lab[t] = m;
            if (!__syncthreads_or(changed)) break;
        }
        if (in) *w.gwp(i, G_REGION) = fluid ? lab[t] : i;
        __syncthreads();
    }
}
// cgJoin's edges between blocks (to the right and below, from the block's
// last column and row), after k_cgStartLocal has linked each block's own.
__global__ void k_cgJoinAcross(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        const int lx = (int)(threadIdx.x & 7u), ly = (int)(threadIdx.x >> 3);
        if (lx != 7 && ly != 7) continue;
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c) || w.gridAt(c).z <= 0.0f) continue;
        for (int d = 0; d < 2; d++) {
            if ((d == 0 && lx != 7) || (d == 1 && ly != 7)) continue;
            I2 n = d == 0 ? I2{c.x + 1, c.y} : I2{c.x, c.y + 1};
            if (rhoAt(w, 0, n) > 0.0f) ufJoin(w, w.cellIndex(c), w.cellIndex(n));
        }
    }
}
// cgAnchor (fluid.wgsl:2692-2705)
__global__ void k_cgAnchor(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c) || w.gridAt(c).z <= 0.0f) continue;
        for (int d = 0; d < 4; d++) {
            I2 n = beside(c, d);
            if (w.inWorld(n) && rhoAt(w, 0, n) == 0.0f) {
                atomicOr(w.gwp(ufFind(w, w.cellIndex(c)), G_REGION), REGION_OPEN);
                break;
            }
        }
    }
}

// FP64 tree of 64 (a block's cells) in shared memory; the sum is in s[0].
__device__ __forceinline__ void tree64(double* s) {
    __syncthreads();
    for (int h = 32; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + h];
        __syncthreads();
    }
}

// cgResidual (fluid.wgsl:2708-2717); with the tolerance form, each block's
// ||b||^2 partial too.
__global__ void k_cgResidual(Dev D) {
    W w(D);
    __shared__ double sb[64];
    const bool tol = D.st->tol_mode != 0u;
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        double b2 = 0.0;
        if (w.inWorld(c) && w.gridAt(c).z > 0.0f) {
            uint32_t i = w.cellIndex(c);
            D.cg[4u * (size_t)i + 1u] = -residualAt(w, 0, c).x - couplingAt(w, c, PUSH_X);
            double b = (double)w.fv(2u * i)[1];
            b2 = b * b;
        }
        if (tol) {
            sb[threadIdx.x] = b2;
            tree64(sb);
            if (threadIdx.x == 0) D.norm64[2u * w.blockIndex(w.activeBlock(wid))] = sb[0];
            __syncthreads();
        }
    }
}
// cgPrepare (fluid.wgsl:2721-2732)
__global__ void k_cgPrepare(Dev D) {
    W w(D);
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        w.fv(2u * i)[0] = 0.0f;
        if (w.fv(2u * i)[2] > 0.0f) w.fv(2u * i)[1] = -D.cg[4u * (size_t)i + 1u];
    }
}

// One CTA of 256: the active blocks' FP64 partials (component comp of 2 in
// buf) summed in sumBlocks' order; the result in the returned value on
// thread 0.
__device__ double sumBlocks64(const W& w, const double* buf, int comp, double* s) {
    double acc = 0.0;
    const uint32_t B = w.D.B;
    for (uint32_t k0 = threadIdx.x; k0 < B; k0 += 256u * 16u) {
        double v[16];
        uint32_t st[16];
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const uint32_t k = k0 + 256u * (uint32_t)u;
            st[u] = k < B ? w.D.blocks[w.stateSlot(k)] : 0u;
            v[u] = k < B ? buf[2u * k + (uint32_t)comp] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; u++)
            if ((st[u] & ACTIVE) != 0u) acc = acc + v[u];
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + h];
        __syncthreads();
    }
    double r = s[0];
    __syncthreads();
    return r;
}

// ||b||^2 of the tolerance form (after cgResidual), and ||r||/||b|| (after
// cgUpdate): one CTA of 256.
__global__ void __launch_bounds__(256) k_norm(Dev D, int which, uint32_t cycle) {
    W w(D);
    __shared__ double s[256];
    if (which == 1 && w.converged(cycle)) return;
    double v = sumBlocks64(w, D.norm64, 0, s);
    if (threadIdx.x == 0) {
        if (which == 0) {
            D.st->bnorm2 = v;
            D.st->rel = 1.0;
        } else {
            D.st->rel = D.st->bnorm2 > 0.0 ? sqrt(v / D.st->bnorm2) : 0.0;
        }
    }
}

// ================================================================ relaxation

// relaxRims (fluid.wgsl:2096-2107)
__global__ void k_relaxRims(Dev D, uint32_t cycle) {
    W w(D);
    if (w.converged(cycle)) return;
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        float4 g = w.f4(2u * i);
        if (g.z > 0.0f) {
            *w.gwp(i, G_RIM) = __float_as_uint(g.x);
            *w.gwp(i, G_RIM + 1u) = __float_as_uint(w.fv(2u * i + 1u)[0]);
        }
    }
}

// tileBlock (fluid.wgsl:2080-2091)
__device__ I2 tileBlock(const W& w, uint32_t wid, int shift) {
    if (wid < w.activeCount()) return w.activeBlock(wid);
    int wide = (int)w.D.BW, high = (int)w.D.BH;
    int j = (int)wid - (int)w.D.B;
    if (shift == 0 || j < 0 || j > high + wide) return I2{-1, -1};
    return j <= high ? I2{wide, j} : I2{j - high - 1, high};
}

// relax / relaxShifted (fluid.wgsl:2109-2192): a CTA per tile, the tile's
// pressure and drift in shared memory for 4 red-black sweep pairs.  The
// tiles are the active blocks' (workgroups [0, activeCount)) and, shifted,
// the edge tiles (workgroups [B, B + edge_tiles)); the grid strides over
// both ranges.
__global__ void __launch_bounds__(64) k_relax(Dev D, int shift, uint32_t cycle) {
    W w(D);
    __shared__ float tpx[RIM * RIM], tpy[RIM * RIM], trho[RIM * RIM], tshare[RIM * RIM];
    __shared__ int s_live, s_ox, s_oy;
    if (w.converged(cycle)) return;
    const uint32_t na = w.activeCount();
    const uint32_t total = na + (shift ? D.edge_tiles : 0u);
    for (uint32_t j = blockIdx.x; j < total; j += gridDim.x) {
        uint32_t wid = j < na ? j : D.B + (j - na);
        if (threadIdx.x == 0) {
            I2 b = tileBlock(w, wid, shift);
            int ox = b.x * BLOCK - shift, oy = b.y * BLOCK - shift;
            uint32_t live = 0;
            if (b.x >= 0 && ox < D.W && oy < D.H)
                live = w.statesOf(I2{ox / BLOCK, oy / BLOCK}, I2{(ox + BLOCK - 1) / BLOCK, (oy + BLOCK - 1) / BLOCK}) & HAS_FLUID;
            s_live = (int)live;
            s_ox = ox;
            s_oy = oy;
        }
        __syncthreads();
        if (s_live) {
            const int ox = s_ox, oy = s_oy;
            for (int k = (int)threadIdx.x; k < RIM * RIM; k += 64) {
                I2 c{ox - 1 + k % RIM, oy - 1 + k / RIM};
                float px = 0.0f, py = 0.0f, rho = -1.0f;
                if (w.inWorld(c)) {
                    uint32_t i = w.cellIndex(c);
                    float4 g = w.f4(2u * i);
                    px = g.x;
                    py = w.fv(2u * i + 1u)[0];
                    rho = g.z;
                    if (rho > 0.0f) {
                        px = __uint_as_float(w.gw(i, G_RIM));
                        py = __uint_as_float(w.gw(i, G_RIM + 1u));
                    }
                }
                tpx[k] = px;
                tpy[k] = py;
                trho[k] = rho;
                tshare[k] = w.densityAt(c);
            }
            __syncthreads();
            const int lx = (int)(threadIdx.x & 7u), ly = (int)(threadIdx.x >> 3);
            I2 me{ox + lx, oy + ly};
            const int t = (ly + 1) * RIM + lx + 1;
            float rho = trho[t];
            float rx = 0.0f, ry = 0.0f, bx = 0.0f, by = 0.0f, bz = 0.0f, bw = 0.0f;
            uint32_t idx = 0;
            if (rho > 0.0f) {
                idx = w.cellIndex(me);
                rx = w.fv(2u * idx)[1];
                ry = w.fv(2u * idx + 1u)[1];
                float d = tshare[t];
                bx = fineBeta(rho, trho[t - 1], d, tshare[t - 1]);
                by = fineBeta(rho, trho[t + 1], d, tshare[t + 1]);
                bz = fineBeta(rho, trho[t - RIM], d, tshare[t - RIM]);
                bw = fineBeta(rho, trho[t + RIM], d, tshare[t + RIM]);
            }
            float diag = bx + by + bz + bw;
            bool pinned = rho > 0.0f && pinnedAt(w, idx);
            float dx = diag + (pinned ? PIN : 0.0f), dy = fmaxf(diag, 1e-30f);
            bool solving = dx > 0.0f;
            int color = (me.x + me.y) & 1;
            for (int sw = 0; sw < 2 * SWEEPS; sw++) {
                if (solving && color == (sw & 1)) {
                    float sx = bx * tpx[t - 1] + by * tpx[t + 1] + bz * tpx[t - RIM] + bw * tpx[t + RIM];
                    float sy = bx * tpy[t - 1] + by * tpy[t + 1] + bz * tpy[t - RIM] + bw * tpy[t + RIM];
                    float nx = mixf(tpx[t], (sx - rx) / dx, SMOOTH_OMEGA);
                    float ny = mixf(tpy[t], (sy - ry) / dy, SMOOTH_OMEGA);
                    tpx[t] = nx;
                    if (diag > 0.0f) tpy[t] = ny;
                }
                __syncthreads();
            }
            if (solving) {
                w.fv(2u * idx)[0] = tpx[t];
                w.fv(2u * idx + 1u)[0] = tpy[t];
            }
        }
        __syncthreads();
    }
}

// ================================================================ multigrid

// restrictLevel (fluid.wgsl:2342-2377): a thread per coarse cell.
__global__ void k_restrict(Dev D, uint32_t l, uint32_t cycle) {
    W w(D);
    I2 c{(int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(blockIdx.y * blockDim.y + threadIdx.y)};
    if (!inLevel(D, l, c) || w.activeCount() == 0u || w.converged(cycle)) return;
    uint32_t at = levelSlot(D, l, c);
    float4* F4 = reinterpret_cast<float4*>(D.field);
    int span = 1 << l;
    if (span <= BLOCK) {
        I2 b{c.x * span / BLOCK, c.y * span / BLOCK};
        if (w.inBlocks(b) && (D.blocks[w.stateSlot(w.blockIndex(b))] & ACTIVE) == 0u) {
            F4[at] = make_float4(0, 0, 0, 0);
            F4[at + 1u] = make_float4(0, 0, 0, 0);
            return;
        }
    }
    float fluid = 0.0f, sum = 0.0f;
    bool air = false;
    V2 r{0.0f, 0.0f};
    for (int j = 0; j < 4; j++) {
        I2 k{2 * c.x + (j & 1), 2 * c.y + (j >> 1)};
        float rho = rhoAt(w, l - 1u, k);
        if (rho == 0.0f) air = true;
        else if (rho > 0.0f) {
            fluid = fluid + 1.0f;
            sum = sum + rho;
            V2 rr = residualAt(w, l - 1u, k);
            r.x = r.x + rr.x;
            r.y = r.y + rr.y;
        }
    }
    float rho = air ? 0.0f : (fluid > 0.0f ? sum / fluid : -1.0f);
    F4[at] = make_float4(0.0f, 0.0f, rho > 0.0f ? r.x * 0.25f : 0.0f, rho > 0.0f ? r.y * 0.25f : 0.0f);
    F4[at + 1u] = make_float4(rho, 0.0f, 0.0f, 0.0f);
}

// smoothRed / smoothBlack (smoothAt, fluid.wgsl:2318-2334, :2379-2387)
__global__ void k_smooth(Dev D, uint32_t l, int color, uint32_t cycle) {
    W w(D);
    I2 c{(int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(blockIdx.y * blockDim.y + threadIdx.y)};
    if (!inLevel(D, l, c) || ((c.x + c.y) & 1) != color || w.activeCount() == 0u || w.converged(cycle)) return;
    uint32_t at = levelSlot(D, l, c);
    float rho = w.fv(at + 1u)[0];
    if (rho <= 0.0f) return;
    V2 sum;
    float diag;
    stencil(w, l, c, rho, &sum, &diag);
    if (diag <= 0.0f) return;
    float* e = w.fv(at);
    float h2 = (float)(1u << (2u * l));
    float sx = (sum.x - h2 * e[2]) / diag, sy = (sum.y - h2 * e[3]) / diag;
    e[0] = mixf(e[0], sx, 1.0f);
    e[1] = mixf(e[1], sy, 1.0f);
}

// solve (fluid.wgsl:2407-2456): the coarsest level (<= 512 cells) in one
// CTA's shared memory, 40 red-black SOR sweep pairs; a thread per cell.
__global__ void __launch_bounds__(512) k_solve(Dev D, uint32_t l, uint32_t cycle) {
    W w(D);
    __shared__ float px[WIG_MG_COARSEST], py[WIG_MG_COARSEST], rx[WIG_MG_COARSEST], ry[WIG_MG_COARSEST], rh[WIG_MG_COARSEST];
    if (w.converged(cycle)) return;
    const int sx = (int)D.level_w[l], sy = (int)D.level_h[l];
    const uint32_t n = min((uint32_t)(sx * sy), WIG_MG_COARSEST);
    const uint32_t j = threadIdx.x;
    if (j < n) {
        I2 c{(int)(j % (uint32_t)sx), (int)(j / (uint32_t)sx)};
        float4 f = w.f4(levelSlot(D, l, c));
        px[j] = f.x; py[j] = f.y; rx[j] = f.z; ry[j] = f.w;
        rh[j] = w.fv(levelSlot(D, l, c) + 1u)[0];
    }
    __syncthreads();
    const float h2 = (float)(1u << (2u * l));
    const int cx = (int)(j % (uint32_t)sx), cy = (int)(j / (uint32_t)sx);
    for (int s = 0; s < 2 * COARSE_SWEEPS; s++) {
        if (j < n && ((cx + cy) & 1) == (s & 1) && rh[j] > 0.0f) {
            float r0 = rh[j];
            float sumx = 0.0f, sumy = 0.0f, diag = 0.0f;
            for (int d = 0; d < 4; d++) {
                I2 o = beside(I2{cx, cy}, d);
                if (o.x < 0 || o.y < 0 || o.x >= sx || o.y >= sy) continue;
                uint32_t oi = (uint32_t)o.y * (uint32_t)sx + (uint32_t)o.x;
                float r = rh[oi];
                if (r < 0.0f) continue;
                float beta = faceBeta(r0, r);
                sumx = sumx + beta * px[oi];
                sumy = sumy + beta * py[oi];
                diag = diag + beta;
            }
            if (diag > 0.0f) {
                px[j] = mixf(px[j], (sumx - h2 * rx[j]) / diag, OMEGA);
                py[j] = mixf(py[j], (sumy - h2 * ry[j]) / diag, OMEGA);
            }
        }
        __syncthreads();
    }
    if (j < n) {
        I2 c{cx, cy};
        reinterpret_cast<float4*>(D.field)[levelSlot(D, l, c)] = make_float4(px[j], py[j], rx[j], ry[j]);
    }
}

// prolong (fluid.wgsl:2459-2470)
__global__ void k_prolong(Dev D, uint32_t l, uint32_t cycle) {
    W w(D);
    I2 c{(int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(blockIdx.y * blockDim.y + threadIdx.y)};
    if (!inLevel(D, l, c) || w.activeCount() == 0u || w.converged(cycle)) return;
    uint32_t at = levelSlot(D, l, c);
    if (w.fv(at + 1u)[0] > 0.0f) {
        V2 e = prolonged(w, l, c);
        float* f = w.fv(at);
        f[0] = f[0] + e.x;
        f[1] = f[1] + e.y;
    }
}

// prolongFine (fluid.wgsl:2500-2512)
__global__ void k_prolongFine(Dev D, uint32_t cycle) {
    W w(D);
    if (w.converged(cycle)) return;
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = 2u * w.cellIndex(c);
        if (w.fv(i)[2] > 0.0f) {
            V2 e = prolonged(w, 0, c);
            w.fv(i)[0] = w.fv(i)[0] + e.x;
            w.fv(i + 1u)[0] = w.fv(i + 1u)[0] + e.y;
        }
    }
}

// ================================================================ conjugate gradients

// A block's partial sums into its slot (sumBlock, fluid.wgsl:2628-2641): the
// same tree of 64.
__device__ __forceinline__ void sumBlock(const W& w, uint32_t wid, float vx, float vy, float* sx, float* sy) {
    sx[threadIdx.x] = vx;
    sy[threadIdx.x] = vy;
    __syncthreads();
    for (int h = 32; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            sx[threadIdx.x] = sx[threadIdx.x] + sx[threadIdx.x + h];
            sy[threadIdx.x] = sy[threadIdx.x] + sy[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        uint32_t b = w.D.C + w.blockIndex(w.activeBlock(wid));
        reinterpret_cast<float4*>(w.D.cg)[b] = make_float4(sx[0], sy[0], 0.0f, 0.0f);
    }
    __syncthreads();
}
// sumBlocks (fluid.wgsl:2645-2661): one CTA of 256.
__device__ V2 sumBlocks(const W& w, float* sx, float* sy) {
    float ax = 0.0f, ay = 0.0f;
    const uint32_t B = w.D.B;
    for (uint32_t k0 = threadIdx.x; k0 < B; k0 += 256u * 8u) {
        float px[8], py[8];
        uint32_t st[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const uint32_t k = k0 + 256u * (uint32_t)u;
            st[u] = k < B ? w.D.blocks[w.stateSlot(k)] : 0u;
            float4 p = k < B ? reinterpret_cast<const float4*>(w.D.cg)[w.D.C + k] : make_float4(0, 0, 0, 0);
            px[u] = p.x;
            py[u] = p.y;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            if ((st[u] & ACTIVE) != 0u) {
                ax = ax + px[u];
                ay = ay + py[u];
            }
        }
    }
    sx[threadIdx.x] = ax;
    sy[threadIdx.x] = ay;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            sx[threadIdx.x] = sx[threadIdx.x] + sx[threadIdx.x + h];
            sy[threadIdx.x] = sy[threadIdx.x] + sy[threadIdx.x + h];
        }
        __syncthreads();
    }
    return V2{sx[0], sy[0]};
}

// cgRho (fluid.wgsl:2736-2750)
__global__ void __launch_bounds__(64) k_cgRho(Dev D, uint32_t cycle) {
    W w(D);
    __shared__ float sx[64], sy[64];
    __shared__ double dx[64], dy[64];
    if (w.converged(cycle)) return;
    const bool f64 = D.st->f64 != 0u;
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        float vx = 0.0f, vy = 0.0f;
        double ex = 0.0, ey = 0.0;
        if (w.inWorld(c) && w.gridAt(c).z > 0.0f) {
            uint32_t i = w.cellIndex(c);
            float z = w.fv(2u * i)[0];
            float4 g = reinterpret_cast<const float4*>(D.cg)[i];
            vx = g.y * z;
            vy = g.w * z;
            ex = (double)g.y * (double)z;
            ey = (double)g.w * (double)z;
        }
        sumBlock(w, wid, vx, vy, sx, sy);
        if (f64) {
            dx[threadIdx.x] = ex;
            tree64(dx);
            dy[threadIdx.x] = ey;
            tree64(dy);
            if (threadIdx.x == 0) {
                uint32_t b = w.blockIndex(w.activeBlock(wid));
                D.part64[2u * b] = dx[0];
                D.part64[2u * b + 1u] = dy[0];
            }
            __syncthreads();
        }
    }
}

// cgBeta (fluid.wgsl:2752-2764): one CTA of 256.
__global__ void __launch_bounds__(256) k_cgBeta(Dev D, uint32_t cycle) {
    W w(D);
    __shared__ float sx[256], sy[256];
    __shared__ double s64[256];
    if (w.converged(cycle) || w.activeCount() == 0u) return;
    float* at = D.cg + 4u * (size_t)(D.C + D.B);
    if (D.st->f64) {
        double rz = sumBlocks64(w, D.part64, 0, s64);
        double zq = sumBlocks64(w, D.part64, 1, s64);
        if (threadIdx.x == 0) {
            double beta = (cycle == 0u || D.st->pq <= 0.0) ? 0.0 : -zq / D.st->pq;
            D.st->rz = rz;
            D.st->beta = beta;
            at[0] = (float)rz;
            at[2] = (float)beta;
        }
        return;
    }
    V2 s = sumBlocks(w, sx, sy);
    if (threadIdx.x == 0) {
        float4 was = make_float4(at[0], at[1], at[2], at[3]);
        float beta = (cycle == 0u || was.w <= 0.0f) ? 0.0f : -s.y / was.w;
        at[0] = s.x;
        at[1] = was.y;
        at[2] = beta;
        at[3] = was.w;
    }
}

// cgDirection (fluid.wgsl:2767-2776)
__global__ void k_cgDirection(Dev D, uint32_t cycle) {
    W w(D);
    if (w.converged(cycle)) return;
    const float beta = D.cg[4u * (size_t)(D.C + D.B) + 2u];
    const bool f64 = D.st->f64 != 0u;
    const double beta64 = D.st->beta;
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        float* g = D.cg + 4u * (size_t)i;
        float p = 0.0f;
        float4 fc = w.f4(2u * i);
        if (fc.z > 0.0f) p = f64 ? (float)((double)fc.x + beta64 * (double)g[2]) : fc.x + beta * g[2];
        g[2] = p;
    }
}

// applyA (fluid.wgsl:2595-2613)
__device__ float applyA(const W& w, I2 c, float rho) {
    float sum = 0.0f, diag = 0.0f;
    float share = w.densityAt(c);
    for (int d = 0; d < 4; d++) {
        I2 n = beside(c, d);
        float r = rhoAt(w, 0, n);
        if (r < 0.0f) continue;
        float beta = fineBeta(rho, r, share, w.densityAt(n));
        if (r > 0.0f) sum = sum + beta * w.D.cg[4u * (size_t)w.cellIndex(n) + 2u];
        diag = diag + beta;
    }
    diag = diag + (pinnedAt(w, w.cellIndex(c)) ? PIN : 0.0f);
    return diag * w.D.cg[4u * (size_t)w.cellIndex(c) + 2u] - sum;
}

// cgApply (fluid.wgsl:2779-2795)
__global__ void __launch_bounds__(64) k_cgApply(Dev D, uint32_t cycle) {
    W w(D);
    __shared__ float sx[64], sy[64];
    __shared__ double dx[64];
    if (w.converged(cycle)) return;
    const bool f64 = D.st->f64 != 0u;
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        float vx = 0.0f;
        double ex = 0.0;
        if (w.inWorld(c)) {
            float rho = w.gridAt(c).z;
            uint32_t i = w.cellIndex(c);
            float q = rho > 0.0f ? applyA(w, c, rho) + couplingAt(w, c, PUSH_P0 + cycle % 2u) : 0.0f;
            float* g = D.cg + 4u * (size_t)i;
            g[3] = q;
            vx = g[2] * q;
            ex = (double)g[2] * (double)q;
        }
        sumBlock(w, wid, vx, 0.0f, sx, sy);
        if (f64) {
            dx[threadIdx.x] = ex;
            tree64(dx);
            if (threadIdx.x == 0) {
                uint32_t b = w.blockIndex(w.activeBlock(wid));
                D.part64[2u * b] = dx[0];
                D.part64[2u * b + 1u] = 0.0;
            }
            __syncthreads();
        }
    }
}

// cgAlpha (fluid.wgsl:2797-2814): one CTA of 256.
__global__ void __launch_bounds__(256) k_cgAlpha(Dev D, uint32_t cycle) {
    W w(D);
    __shared__ float sx[256], sy[256];
    __shared__ double s64[256];
    if (w.converged(cycle) || w.activeCount() == 0u) return;
    // the bodies' sums of this iteration's direction, done with, emptied for
    // the iteration after next (fluid.wgsl:2808-2813)
    if (D.pushes) {
        const uint32_t which = PUSH_P0 + cycle % 2u;
        for (uint32_t k = threadIdx.x; k < MAX_BODIES * 6u; k += blockDim.x)
            D.pushes[pushSlot(k / 6u, which, 0u) + k % 6u] = 0u;
    }
    float* at = D.cg + 4u * (size_t)(D.C + D.B);
    if (D.st->f64) {
        double pq = sumBlocks64(w, D.part64, 0, s64);
        if (threadIdx.x == 0) {
            D.st->pq = pq;
            D.st->alpha = pq <= 0.0 ? 0.0 : D.st->rz / pq;
            at[1] = (float)D.st->alpha;
            at[3] = (float)pq;
        }
        return;
    }
    float pq = sumBlocks(w, sx, sy).x;
    if (threadIdx.x == 0) {
        float4 was = make_float4(at[0], at[1], at[2], at[3]);
        at[0] = was.x;
        at[1] = pq <= 0.0f ? 0.0f : was.x / pq;
        at[2] = was.z;
        at[3] = pq;
    }
}

// cgUpdate (fluid.wgsl:2852-2880); with the tolerance form, each block's
// ||r||^2 partial too.
__global__ void __launch_bounds__(64) k_cgUpdate(Dev D, uint32_t cycle) {
    W w(D);
    __shared__ uint32_t most;
    __shared__ double sb[64];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        D.blocks[w.countSlot(COUNT_RESIDUAL + (cycle + 1u) % 3u)] = 0u;
        if (!w.converged(cycle)) D.blocks[w.countSlot(COUNT_CYCLES)] += 1u;
    }
    if (w.converged(cycle)) return;
    const float alpha = D.cg[4u * (size_t)(D.C + D.B) + 1u];
    const bool f64 = D.st->f64 != 0u, tol = D.st->tol_mode != 0u;
    const double alpha64 = D.st->alpha;
    FOR_ACTIVE(D, w, wid) {
        if (threadIdx.x == 0) most = 0u;
        __syncthreads();
        I2 c = lidCell(w, wid);
        double r2 = 0.0;
        if (w.inWorld(c) && w.gridAt(c).z > 0.0f) {
            uint32_t i = w.cellIndex(c);
            float4 v = reinterpret_cast<const float4*>(D.cg)[i];
            float r, x;
            if (f64) {
                r = (float)((double)v.y - alpha64 * (double)v.w);
                x = (float)((double)v.x + alpha64 * (double)v.z);
            } else {
                r = v.y - alpha * v.w;
                x = v.x + alpha * v.z;
            }
            reinterpret_cast<float4*>(D.cg)[i] = make_float4(x, r, v.z, v.w);
            w.fv(2u * i)[0] = 0.0f;
            w.fv(2u * i)[1] = -r;
            atomicMax(&most, __float_as_uint(fabsf(r)));
            r2 = (double)r * (double)r;
        }
        if (tol) {
            sb[threadIdx.x] = r2;
            tree64(sb);
            if (threadIdx.x == 0) D.norm64[2u * w.blockIndex(w.activeBlock(wid))] = sb[0];
        }
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(&D.blocks[w.countSlot(COUNT_RESIDUAL + cycle % 3u)], most);
        __syncthreads();
    }
}

// cgFinish (fluid.wgsl:2884-2893)
__global__ void k_cgFinish(Dev D) {
    W w(D);
    FOR_ACTIVE(D, w, wid) {
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        w.fv(2u * i)[0] = D.cg[4u * (size_t)i];
        *w.gwp(i, G_REGION) = 0u;
    }
}

// ================================================================ projection, extrapolation

// project / projectFace (fluid.wgsl:2897-2942)
__global__ void k_project(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    // once a world: the most iterations any step took
    if (threadIdx.x == 0) {
        FOR_ITEMS(Bt, L_ONE, ot) {
            ITEM_WORLD(Bt, ot, D, w, unused_);
            (void)unused_;
            uint32_t cyc = D.blocks[w.countSlot(COUNT_CYCLES)];
            atomicMax(&D.blocks[w.countSlot(COUNT_MOST_CYCLES)], cyc);
        }
    }
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        int fs[4][3];
        w.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            I2 at{fs[j][0], fs[j][1]};
            bool isU = fs[j][2] == 1;
            float4* fp = reinterpret_cast<float4*>(D.field) + w.faceSlot(w.faceIndex(at, isU));
            I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
            float4 ga = w.gridAt(a), gb = w.gridAt(at);
            float beta = fineBeta(ga.z, gb.z, w.densityAt(a), w.densityAt(at));
            const uint32_t ra = rigidAt(w, a), rb = rigidAt(w, at);
            if (beta > 0.0f) {
                float4 face = *fp;
                face.x = face.x - beta * (gb.x - ga.x);
                face.z = PROJECTED;
                const bool rigid = ra != NONE || rb != NONE;
                face.w = rigid ? 0.0f : clampf(-beta * (w.driftAt(at) - w.driftAt(a)), -MAX_DRIFT, MAX_DRIFT);
                *fp = face;
            }
            // a face between the liquid and a free body moves with the body's push (PUSH_F)
            if ((ra == NONE) != (rb == NONE) && (ra != NONE ? gb.z : ga.z) > 0.0f) {
                const uint32_t bb = ra != NONE ? ra : rb;
                const V3 ch = pushChange(w, bb, PUSH_F);
                const V2 m = faceMiddle(at, isU), pos = bodyV(w, bb, WIG_BW_POS);
                const V2 r{m.x - pos.x, m.y - pos.y};
                float4 face = *fp;
                face.x = face.x + (isU ? ch.x - ch.z * r.y : ch.y + ch.z * r.x);
                face.z = PROJECTED;
                *fp = face;
            }
        }
    }
}

// extrapolate / extrapolateFurther (fluid.wgsl:3226-3275)
__global__ void k_extrapolate(Batch Bt, uint32_t layer) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        int fs[4][3];
        w.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            I2 at{fs[j][0], fs[j][1]};
            bool isU = fs[j][2] == 1;
            float* face = w.fv(w.faceSlot(w.faceIndex(at, isU)));
            I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
            if (face[2] != 1.0f || w.gridAt(a).z != 0.0f || w.gridAt(at).z != 0.0f) continue;
            float reached = layer == 2u ? 1.5f : PROJECTED;
            float sum = 0.0f, n = 0.0f;
            for (int d = 0; d < 4; d++) {
                I2 q = beside(at, d);
                if (!w.faceInWorld(q, isU)) continue;
                float4 g = w.f4(w.faceSlot(w.faceIndex(q, isU)));
                if (g.z >= reached) { sum = sum + g.x; n = n + 1.0f; }
            }
            if (n > 0.0f) {
                face[0] = sum / n;
                face[2] = layer == 2u ? 1.25f : 1.5f;
            }
        }
    }
}

// ================================================================ advect

struct Sample { float now, weight, drift, gx, gy; };
// sampleAxis (fluid.wgsl:3480-3512)
__device__ Sample sampleAxis(const W& w, float sx, float sy, bool isU) {
    float fx0 = floorf(sx), fy0 = floorf(sy);
    int bx = f2i(fx0), by = f2i(fy0);
    float fx = sx - fx0, fy = sy - fy0;
    float ax = 0.0f;
    Sample r{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    int held = 0;
    float gx = 0.0f, gy = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int ox = j & 1, oy = j >> 1;
        float wgt = (ox == 1 ? fx : 1.0f - fx) * (oy == 1 ? fy : 1.0f - fy);
        float dwx = (ox == 1 ? 1.0f : -1.0f) * (oy == 1 ? fy : 1.0f - fy);
        float dwy = (ox == 1 ? fx : 1.0f - fx) * (oy == 1 ? 1.0f : -1.0f);
        I2 at{bx + ox, by + oy};
        if (!w.faceInWorld(at, isU)) continue;
        float4 face = w.f4(w.faceSlot(w.faceIndex(at, isU)));
        r.drift = r.drift + wgt * face.w;
        if (face.z > 0.0f) {
            ax = ax + wgt * face.x;
            r.weight = r.weight + wgt;
            gx = gx + dwx * face.x;
            gy = gy + dwy * face.x;
            held += face.z == PROJECTED ? 1 : 0;
        }
    }
    if (r.weight > 0.0f) r.now = ax / r.weight;
    if (held == 4) { r.gx = gx; r.gy = gy; }
    return r;
}
__device__ __forceinline__ bool isObstacle(const W& w, float px, float py) {
    I2 c{f2i(floorf(px)), f2i(floorf(py))};
    if (w.gridAt(c).z < 0.0f) return true;
    uint32_t k = w.kindOfCell(w.cellIndex(c));
    return k == WIG_KIND_SOLID || k == WIG_KIND_POWDER;
}
// shutAt, escapesTo (fluid.wgsl:1468-1470, :3535-3541)
__device__ __forceinline__ bool escapesTo(const W& w, I2 q, uint32_t side) {
    if (!w.inWorld(q) || w.gridAt(q).z < 0.0f || rigidAt(w, q) != NONE) return false;
    const uint32_t cup = cupOf(w, w.cellIndex(q));
    return cup == NONE || cup == side;
}
// escape (fluid.wgsl:3552-3594), no bodies, the Earth's down.
__device__ V2 escape(const W& w, V2 pos) {
    if (!isObstacle(w, pos.x, pos.y)) return pos;
    I2 c{f2i(floorf(pos.x)), f2i(floorf(pos.y))};
    const uint32_t side = w.inWorld(c) ? cupBefore(w, w.cellIndex(c)) : NONE;
    V2 best = pos;
    float bestD = 1e9f;
    for (int n = 0; n < 8; n++) {
        int m = n + (n >= 4 ? 1 : 0);
        I2 at{c.x + m % 3 - 1, c.y + m / 3 - 1};
        if (!escapesTo(w, at, side)) continue;
        float ix = clampf(pos.x, (float)at.x + 0.02f, (float)at.x + 0.98f);
        float iy = clampf(pos.y, (float)at.y + 0.02f, (float)at.y + 0.98f);
        float d = len2(pos.x - ix, pos.y - iy);
        if (d < bestD) { bestD = d; best = V2{ix, iy}; }
    }
    if (bestD < 1e9f) return best;
    const int wx[4] = {0, -1, 1, 0}, wy[4] = {-1, 0, 0, 1};
    int wayx = wx[0], wayy = wy[0];
    int nearest = ESCAPE_REACH + 1;
    for (int n = 0; n < 4; n++) {
        for (int r = 2; r < nearest; r++) {
            I2 q{c.x + wx[n] * r, c.y + wy[n] * r};
            if (!isObstacle(w, (float)q.x + 0.5f, (float)q.y + 0.5f) && escapesTo(w, q, side)) {
                nearest = r;
                wayx = wx[n];
                wayy = wy[n];
                break;
            }
        }
    }
    return w.inWorld(I2{c.x + wayx, c.y + wayy}) ? V2{pos.x + (float)wayx, pos.y + (float)wayy} : pos;
}
__device__ __forceinline__ V2 clampSpeed(V2 v) {
    float s = len2(v.x, v.y);
    if (s > LIQUID_MAX_SPEED) {
        float k = LIQUID_MAX_SPEED / s;
        return V2{v.x * k, v.y * k};
    }
    return v;
}

// advect (fluid.wgsl:3616-3694)
__device__ __forceinline__ void advectOne(const Dev& D, const W& w, uint32_t chunk) {
    uint32_t live = min(D.parts[0], D.cap);
    uint32_t k = chunk * blockDim.x + threadIdx.x;
    if (k >= live) return;
    uint4* it = w.items(D.parts);
    uint4 mo = it[k], stt = it[D.cap + k];
    V2 orig{__uint_as_float(mo.x), __uint_as_float(mo.y)};
    V2 qvel{__uint_as_float(mo.z), __uint_as_float(mo.w)};
    float temp = __uint_as_float(stt.y);
    V2 qpos = escape(w, orig);
    Sample u = sampleAxis(w, qpos.x - 0.0f, qpos.y - 0.5f, true);
    Sample v = sampleAxis(w, qpos.x - 0.5f, qpos.y - 0.0f, false);
    V2 flow{u.weight > 0.0f ? u.now : qvel.x, v.weight > 0.0f ? v.now : qvel.y};
    V2 vel = clampSpeed(flow);
    float4 affine = make_float4(AFFINE_KEEP * u.gx, AFFINE_KEEP * u.gy, AFFINE_KEEP * v.gx, AFFINE_KEEP * v.gy);
    V2 cs = clampSpeed(vel);
    // slipOf (fluid.wgsl:3605-3614)
    V2 sl{0.0f, 0.0f};
    {
        uint32_t i = w.cellIndex(w.cellOf(qpos.x, qpos.y));
        uint32_t n = w.gw(i, G_COUNT);
        if (n >= 2u) {
            float mean = (float)w.gw(i, G_MASS) / (FIX * (float)n);
            float lighter = (mean - w.liquidDensity(stt.x, temp)) / fmaxf(mean, 1e-3f);
            V2 pl = w.pull();
            float wgt = w.elem(WATER).weight;
            sl = V2{-pl.x / wgt * SLIP * lighter, -pl.y / wgt * SLIP * lighter};
        }
    }
    V2 travel{cs.x + clampf(u.drift + sl.x, -MAX_DRIFT, MAX_DRIFT), cs.y + clampf(v.drift + sl.y, -MAX_DRIFT, MAX_DRIFT)};
    int steps = min(max(f2i(ceilf(fmaxf(fabsf(travel.x), fabsf(travel.y)) * 2.0f)), 1), ADVECT_STEPS);
    float dx = travel.x / (float)steps, dy = travel.y / (float)steps;
    V2 pos = qpos;
    float impact = 0.0f;
    for (int s = 0; s < steps; s++) {
        float nx = pos.x + dx, nxy = pos.y + 0.0f;
        if (dx != 0.0f && isObstacle(w, nx, nxy)) {
            if (vel.x * dx > 0.0f) { impact = fmaxf(impact, fabsf(vel.x)); vel.x = 0.0f; }
            dx = 0.0f;
        } else {
            pos = V2{nx, nxy};
        }
        float nyx = pos.x + 0.0f, ny = pos.y + dy;
        if (dy != 0.0f && isObstacle(w, nyx, ny)) {
            if (vel.y * dy > 0.0f) { impact = fmaxf(impact, fabsf(vel.y)); vel.y = 0.0f; }
            dy = 0.0f;
        } else {
            pos = V2{nyx, ny};
        }
    }
    {
        I2 pc = w.cellOf(pos.x, pos.y);
        if (!w.isActiveBlock(I2{pc.x / BLOCK, pc.y / BLOCK})) {
            pos = qpos;
            I2 qc = w.cellOf(pos.x, pos.y);
            if (!w.isActiveBlock(I2{qc.x / BLOCK, qc.y / BLOCK})) pos = orig;
        }
    }
    it[k] = make_uint4(__float_as_uint(pos.x), __float_as_uint(pos.y), __float_as_uint(vel.x), __float_as_uint(vel.y));
    it[2u * D.cap + k] = make_uint4(__float_as_uint(affine.x), __float_as_uint(affine.y), __float_as_uint(affine.z),
                                    __float_as_uint(affine.w));
    float4 left = w.f4(2u * w.cellIndex(w.cellOf(qpos.x, qpos.y)));
    if (left.z > 0.0f) {
        V2 pl = w.pull();
        bool falling = left.x < 0.5f * left.z * len2(pl.x, pl.y);
        atomicOr(w.gwp(w.cellIndex(w.cellOf(pos.x, pos.y)), G_CAME), falling ? CAME_FALLING : CAME_PRESSING);
    }
    if ((w.elem(wordType(stt.x)).flags & F_IMPACT) != 0u && impact > IMPACT_SPEED) it[D.cap + k].x = wordWith(stt.x, FL_BURN);
}
__global__ void k_advect(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_PP, qi) {
        ITEM_WORLD_C(Bt, qi, D, w, chunk);
        advectOne(D, w, chunk);
    }
}

// ================================================================ sort

// sortCount (fluid.wgsl:3700-3708): each particle's slot among its cell's.
// The lanes of a warp whose particles share a cell (parts is in cell order
// from the last sort, so mostly neighbours) take their slots with one atomic
// add by the lowest of them, each lane its rank among them past the base;
// the slots within a cell are any order of 0..n-1, as the reference's
// atomics give them.
__device__ __forceinline__ void sortCountOne(const Dev& D, const W& w, uint32_t chunk) {
    uint32_t live = min(D.parts[0], D.cap);
    uint32_t k = chunk * blockDim.x + threadIdx.x;
    if (k >= live) return;
    uint4* it = w.items(D.parts);
    uint4 mo = it[k];
    uint32_t i = w.cellIndex(w.cellOf(__uint_as_float(mo.x), __uint_as_float(mo.y)));
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t peers = __match_any_sync(__activemask(), i);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0u;
    if ((int)lane == leader) base = atomicAdd(w.gwp(i, G_SORT), (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    it[D.cap + k].w = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}
__global__ void k_sortCount(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_PP, qi) {
        ITEM_WORLD_C(Bt, qi, D, w, chunk);
        sortCountOne(D, w, chunk);
    }
}

// scanBlocks (fluid.wgsl:3730-3753)
__global__ void __launch_bounds__(64) k_scanBlocks(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    __shared__ uint32_t tile[64];
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        const uint32_t fall0 = 4u << (D.st->P.frame & 1u);
        I2 c = lidCell(w, wid);
        uint32_t n = 0;
        if (w.inWorld(c)) n = w.gw(w.cellIndex(c), G_SORT);
        tile[threadIdx.x] = n;
        __syncthreads();
        for (uint32_t o = 1; o < 64u; o <<= 1) {
            uint32_t add = threadIdx.x >= o ? tile[threadIdx.x - o] : 0u;
            __syncthreads();
            tile[threadIdx.x] += add;
            __syncthreads();
        }
        if (w.inWorld(c)) {
            uint32_t i = w.cellIndex(c);
            *w.gwp(i, G_START) = tile[threadIdx.x] - n;
            uint32_t came = atomicExch(w.gwp(i, G_CAME), 0u);
            if (came == CAME_FALLING) {
                float* fw = w.fv(2u * i + 1u) + 3;
                *fw = (float)(f2u(*fw) | fall0);
            }
        }
        if (threadIdx.x == 63u) D.blocks[w.totalSlot(wid)] = tile[63];
        __syncthreads();
    }
}

// scanTotals (fluid.wgsl:3757-3780): one CTA of 256.
__global__ void __launch_bounds__(256) k_scanTotals(Batch Bt) {
  __shared__ uint32_t tile[256];
  FOR_ITEMS(Bt, L_ONE, ot) {
    ITEM_WORLD(Bt, ot, D, w, unused_);
    (void)unused_;
    const uint32_t n = w.activeCount();
    const uint32_t per = (n + 255u) / 256u;
    const uint32_t lo = min(threadIdx.x * per, n), hi = min(lo + per, n);
    uint32_t sum = 0;
    for (uint32_t j = lo; j < hi; j++) sum += D.blocks[w.totalSlot(j)];
    tile[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t o = 1; o < 256u; o <<= 1) {
        uint32_t add = threadIdx.x >= o ? tile[threadIdx.x - o] : 0u;
        __syncthreads();
        tile[threadIdx.x] += add;
        __syncthreads();
    }
    uint32_t run = tile[threadIdx.x] - sum;
    for (uint32_t j = lo; j < hi; j++) {
        uint32_t t = D.blocks[w.totalSlot(j)];
        D.blocks[w.totalSlot(j)] = run;
        run += t;
    }
    if (threadIdx.x == 255u) {
        D.sorted[0] = tile[255];
        D.blocks[w.countSlot(COUNT_PARTICLES)] = tile[255];
    }
    __syncthreads();
  }
}

// scanFinish (fluid.wgsl:3783-3790)
__global__ void k_scanFinish(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        *w.gwp(w.cellIndex(c), G_START) += D.blocks[w.totalSlot(wid)];
    }
}

// scatter (fluid.wgsl:3793-3808)
__device__ __forceinline__ void scatterOne(const Dev& D, const W& w, uint32_t chunk) {
    uint32_t live = min(D.parts[0], D.cap);
    uint32_t k = chunk * blockDim.x + threadIdx.x;
    if (k >= live) return;
    const uint4* it = w.items(D.parts);
    uint4 mo = it[k], stt = it[D.cap + k];
    uint32_t i = w.cellIndex(w.cellOf(__uint_as_float(mo.x), __uint_as_float(mo.y)));
    uint32_t m = w.gw(i, G_START) + stt.w;
    if (m < D.cap) {
        uint4* so = w.items(D.sorted);
        so[m] = mo;
        so[D.cap + m] = stt;
        so[2u * D.cap + m] = it[2u * D.cap + k];
    }
}
__global__ void k_scatter(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_PP, qi) {
        ITEM_WORLD_C(Bt, qi, D, w, chunk);
        scatterOne(D, w, chunk);
    }
}

// ================================================================ raster

__device__ __forceinline__ bool vacated(const W& w, uint32_t j) {
    return w.kindOfCell(j) == WIG_KIND_LIQUID && w.gw(j, G_SORT) == 0u;
}
// airTo (fluid.wgsl:3898-3924)
__device__ uint32_t airTo(const W& w, I2 c, bool gas) {
    if (!gas && w.gridAt(c).z > 0.0f) return NONE;
    const int ax[8] = {0, -1, 1, 0, -1, 1, -1, 1}, ay[8] = {-1, 0, 0, 1, -1, -1, 1, 1};
    const int gx[8] = {0, -1, 1, -1, 1, -1, 1, 0}, gy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
    for (int n = 0; n < 8; n++) {
        I2 at{c.x + (gas ? gx[n] : ax[n]), c.y + (gas ? gy[n] : ay[n])};
        if (!w.inWorld(at)) continue;
        uint32_t j = w.cellIndex(at);
        if (vacated(w, j) || (gas && w.cellType(j) == AIR && w.gw(j, G_SORT) == 0u)) return j;
    }
    return NONE;
}
// rasterClaims (fluid.wgsl:3928-3948), no people.
__global__ void k_rasterClaims(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        uint32_t to = NONE;
        uint32_t t = w.cellType(i);
        if (w.gw(i, G_SORT) > 0u) {
            if (t == AIR) to = airTo(w, c, false);
            else if (w.kindOf(t) == WIG_KIND_GAS && w.gridAt(c).z >= 0.0f) to = airTo(w, c, true);
        }
        *w.gwp(i, G_AIR_TO) = to;
        if (to != NONE) atomicMax(w.gwp(to, G_TAKEN), takenBy(i));
    }
}

// exactParts(x, EXACT_FINE) added to a 64-bit sum (common.wgsl:1383-1393,
// fluid.wgsl:4127-4131).
__device__ __forceinline__ unsigned long long exact_add(unsigned long long wsum, float x) {
    float s = rnd_even(clampf(x * EXACT_FINE, -9.2e18f, 9.2e18f));
    uint32_t lo, hi;
    if (fabsf(s) < 2147483648.0f) {
        int32_t v = (int32_t)s;
        lo = (uint32_t)v;
        hi = v < 0 ? 0xffffffffu : 0u;
    } else {
        float h = floorf(s / 4294967296.0f);
        lo = f2u(s - h * 4294967296.0f);
        hi = (uint32_t)f2i(h);
    }
    uint32_t wl = (uint32_t)wsum, wh = (uint32_t)(wsum >> 32);
    uint32_t nl = wl + lo;
    uint32_t nh = wh + hi + (nl < lo ? 1u : 0u);
    return ((unsigned long long)nh << 32) | nl;
}
__device__ __forceinline__ float exact_value(unsigned long long wsum, float scale) {
    int32_t l = (int32_t)(uint32_t)wsum, h = (int32_t)(uint32_t)(wsum >> 32);
    if ((h == 0 && l >= 0) || (h == -1 && l < 0)) return (float)l / scale;
    return ((float)h * 4294967296.0f + (float)(uint32_t)wsum) / scale;
}

// raster (fluid.wgsl:3983-4119), no people, the air source unbound.
__global__ void k_raster(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, qi) {
        ITEM_WORLD_C(Bt, qi, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        uint32_t n = w.gw(i, G_SORT);
        if (n == 0u) continue;
        uint32_t start = w.gw(i, G_START);
        uint4 v = w.cell(i);
        uint32_t t = wordType(v.x);
        bool drawn = false;
        if (w.kindOf(t) == WIG_KIND_LIQUID) {
            drawn = true;
        } else if (t == AIR || (w.kindOf(t) == WIG_KIND_GAS && w.gridAt(c).z >= 0.0f)) {
            uint32_t to = w.gw(i, G_AIR_TO);
            if (to != NONE && to < D.C && w.gw(to, G_TAKEN) == takenBy(i)) {
                if (w.cellType(to) == AIR) {
                    uint32_t* gp = w.gasPairPtr(to);
                    gp[0] = 0u; gp[1] = 0u;
                }
                reinterpret_cast<uint4*>(D.cells)[to] = v;
                uint32_t* gi = w.gasPairPtr(i);
                uint32_t* gt = w.gasPairPtr(to);
                gt[0] = gi[0]; gt[1] = gi[1];
                gi[0] = 0u; gi[1] = 0u;
                drawn = true;
            } else if (t == AIR) {
                uint32_t* gp = w.gasPairPtr(i);
                gp[0] = 0u; gp[1] = 0u;
                drawn = true;
            }
        }
        if (!drawn) {
            *w.gwp(i, G_DEST) = DEST_KEEP;
            continue;
        }
        const uint4* it = w.items(D.sorted);
        uint32_t kinds[RASTER_KINDS] = {NONE, NONE, NONE, NONE};
        uint32_t counts[RASTER_KINDS] = {0, 0, 0, 0};
        for (uint32_t k = start; k < start + n && k < D.cap; k++) {
            uint32_t pt = wordType(it[D.cap + k].x);
            uint32_t at = RASTER_KINDS;
            for (uint32_t m = 0; m < RASTER_KINDS; m++)
                if (kinds[m] == pt) at = m;
            if (at == RASTER_KINDS && pt < kinds[RASTER_KINDS - 1u]) {
                at = RASTER_KINDS - 1u;
                kinds[at] = pt;
                counts[at] = 0u;
                while (at > 0u && kinds[at - 1u] > kinds[at]) {
                    uint32_t t0 = kinds[at - 1u], c0 = counts[at - 1u];
                    kinds[at - 1u] = kinds[at];
                    counts[at - 1u] = counts[at];
                    kinds[at] = t0;
                    counts[at] = c0;
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
        for (uint32_t k = start; k < start + n && k < D.cap; k++) {
            uint4 st = it[D.cap + k];
            if (wordType(st.x) == most && (lowest == NONE || st.z < lowest)) { word = st.x; lowest = st.z; }
            if (solutes && wordType(st.x) == most && wordAux(st.x) != 0u && (soluteId == NONE || st.z < soluteId)) {
                solute = wordAux(st.x);
                soluteId = st.z;
            }
        }
        if (solutes) word = packWord(wordType(word), solute, wordLife(word), wordShade(word), wordFlags(word));
        float lx = 0.0f, ly = 0.0f;
        unsigned long long heat = 0, capa = 0, vx = 0, vy = 0;
        for (uint32_t k = start; k < start + n && k < D.cap; k++) {
            uint4 st = it[D.cap + k];
            uint32_t pt = wordType(st.x);
            if (pt == most && wordAux(st.x) == wordAux(word)) {
                lx = lx + (float)wordLife(st.x);
                ly = ly + 1.0f;
            } else if (pt == most && solutes && wordAux(st.x) == 0u) {
                ly = ly + 1.0f;
            }
            float hc = fmaxf(w.elem(pt).heat_cap, 1e-6f);
            heat = exact_add(heat, hc * __uint_as_float(st.y));
            capa = exact_add(capa, hc);
            uint4 mo = it[k];
            vx = exact_add(vx, __uint_as_float(mo.z));
            vy = exact_add(vy, __uint_as_float(mo.w));
        }
        Rng g;
        g.seed(i, D.st->P.frame, D.st->P.seed ^ 0x7a57u);
        uint32_t life = min(f2u(floorf(lx / ly + g.next())), 255u);
        word = packWord(wordType(word), wordAux(word), life, wordShade(word), wordFlags(word));
        float temp = exact_value(heat, EXACT_FINE) / exact_value(capa, EXACT_FINE);
        float velx = exact_value(vx, EXACT_FINE) / (float)n, vely = exact_value(vy, EXACT_FINE) / (float)n;
        reinterpret_cast<uint4*>(D.cells)[i] = make_uint4(wordWith(word, FL_DRAWN), __float_as_uint(temp), pack2x16(velx, vely), liquidW(i, n));
        *w.gwp(i, G_TYPE) = drawnAs(word) | (life << 16u);
    }
}

// unpaint (fluid.wgsl:4163-4182)
__global__ void k_unpaint(Batch Bt) {
    __shared__ WorldCopy wc_;
    worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        ITEM_WORLD_C(Bt, it, D, w, wid);
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        uint4 v = w.cell(i);
        if (w.kindOf(wordType(v.x)) == WIG_KIND_LIQUID && w.gw(i, G_SORT) == 0u && w.gw(i, G_TAKEN) == 0u) {
            float t = w.actsAt(v.x, __uint_as_float(v.y));
            reinterpret_cast<uint4*>(D.cells)[i] = make_uint4(AIR, __float_as_uint(t), 0u, 0u);
            uint32_t* gp = w.gasPairPtr(i);
            gp[0] = 0u; gp[1] = 0u;
        }
    }
}

// ================================================================ launch

// ================================================================ the bodies' passes (world 0)

// bodyStart (fluid.wgsl:3079-3084)
__global__ void k_bodyStart(Dev D) {
    const uint32_t n = MAX_BODIES * WIG_BODY_PUSH_WORDS;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) D.pushes[k] = 0u;
}

// seepLoads, bodyLoads (fluid.wgsl:3094-3139)
__device__ void seepLoads(const W& w, I2 c, uint32_t b) {
    for (int d = 0; d < 4; d++) {
        const I2 q = beside(c, d);
        if (!w.inWorld(q) || rigidAt(w, q) == b || w.gridAt(q).z >= 0.0f) continue;
        const I2 n{q.x - c.x, q.y - c.y};
        const V2 x{((float)c.x + 0.5f) + 0.5f * (float)n.x, ((float)c.y + 0.5f) + 0.5f * (float)n.y};
        addPush(w, b, PUSH_SURFACE, scale3(bodyFaceJ(w, q, c, b), seepAt(w, c, n, b, false, x)));
    }
}
__global__ void __launch_bounds__(64) k_bodyLoads(Dev D) {
    W w(D);
    FOR_ACTIVE(D, w, wid) {
        const I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        const uint32_t own = rigidAt(w, c);
        if (own != NONE) {
            seepLoads(w, c, own);
            continue;
        }
        const float4 g = w.gridAt(c);
        if (g.z <= 0.0f) continue;
        const V2 mid{(float)c.x + 0.5f, (float)c.y + 0.5f};
        for (int d = 0; d < 4; d++) {
            const I2 q = beside(c, d);
            const uint32_t b = rigidAt(w, q);
            if (b == NONE) continue;
            const I2 n{q.x - c.x, q.y - c.y};
            const float reach = 1.0f - bodyReach(w, b, I2{-n.x, -n.y});
            const V2 surface{mid.x + (float)n.x * reach, mid.y + (float)n.y * reach};
            addPush(w, b, PUSH_SURFACE,
                    scale3(scale3(bodyFaceJ(w, c, q, b), g.z), potentialAt(w, mid) - potentialAt(w, surface)));
        }
    }
}

// bodyDrag (fluid.wgsl:3149-3176)
__global__ void __launch_bounds__(64) k_bodyDrag(Dev D) {
    W w(D);
    FOR_ACTIVE(D, w, wid) {
        const I2 c = lidCell(w, wid);
        const uint32_t b = rigidAt(w, c);
        if (!w.inWorld(c) || b == NONE) continue;
        const V2 pos = bodyV(w, b, WIG_BW_POS);
        const float rho = bodyDensity(w, b);
        V3 push{0.0f, 0.0f, 0.0f};
        for (int k = 0; k < 4; k++) {
            const bool isU = k < 2;
            const int sg = (k & 1) == 1 ? 1 : -1;
            const I2 n = isU ? I2{sg, 0} : I2{0, sg};
            if (w.gridAt(I2{c.x + n.x, c.y + n.y}).z <= 0.0f) continue;
            const I2 at = isU ? I2{c.x + (k & 1), c.y} : I2{c.x, c.y + (k & 1)};
            const V2 x = faceMiddle(at, isU);
            const V2 mv = bodyMoving(w, b, x, false);
            const float du = (bodyReach(w, b, n) * rho) * (w.fv(w.faceSlot(w.faceIndex(at, isU)))[0] - (isU ? mv.x : mv.y));
            const V2 r{x.x - pos.x, x.y - pos.y};
            if (isU) push.x = push.x + du;
            else push.y = push.y + du;
            push.z = push.z + (isU ? -r.y * du : r.x * du);
        }
        if (push.x != 0.0f || push.y != 0.0f || push.z != 0.0f) addPush(w, b, PUSH_DRAG, push);
    }
}

// bodyFaces (fluid.wgsl:3180-3200)
__global__ void __launch_bounds__(64) k_bodyFaces(Dev D) {
    W w(D);
    FOR_ACTIVE(D, w, wid) {
        const I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        int fs[4][3];
        w.facesOf(c, fs);
        for (int j = 0; j < 4; j++) {
            if (fs[j][2] < 0) continue;
            const I2 at{fs[j][0], fs[j][1]};
            const bool isU = fs[j][2] == 1;
            const I2 a = isU ? I2{at.x - 1, at.y} : I2{at.x, at.y - 1};
            const uint32_t ra = rigidAt(w, a), rb = rigidAt(w, at);
            if (ra != NONE || rb != NONE) setBodyFace(w, w.faceIndex(at, isU), at, isU, w.gridAt(a), w.gridAt(at), ra, rb, true);
        }
    }
}

// cgBodyX, cgBodyP, cgBodyF (fluid.wgsl:2819-2845): the pressure's push on
// the bodies beside each liquid cell, of the solve's start (x), of this
// iteration's direction (p, into the set of the iteration's parity) and of
// the pressure it ends with.
__global__ void __launch_bounds__(64) k_cgBody(Dev D, int which, uint32_t cycle) {
    W w(D);
    if (which == 1 && w.converged(cycle)) return;
    FOR_ACTIVE(D, w, wid) {
        const I2 c = lidCell(w, wid);
        if (!w.inWorld(c) || w.gridAt(c).z <= 0.0f) continue;
        const uint32_t i = w.cellIndex(c);
        if (which == 0) addPressurePush(w, c, D.cg[4u * (size_t)i], PUSH_X);
        else if (which == 1) addPressurePush(w, c, D.cg[4u * (size_t)i + 2u], PUSH_P0 + cycle % 2u);
        else addPressurePush(w, c, w.fv(2u * i)[0], PUSH_F);
    }
}

// rigidify (fluid.wgsl:3033-3076): each block's cells of its lowest held
// body summed in shared memory and added once, the others' straight into
// their bodies' words (integer adds: the totals are the same in any order).
__global__ void __launch_bounds__(64) k_rigidify(Dev D) {
    W w(D);
    __shared__ uint32_t first;
    __shared__ uint32_t sums[3];
    FOR_ACTIVE(D, w, wid) {
        if (threadIdx.x == 0) {
            first = NONE;
            sums[0] = sums[1] = sums[2] = 0u;
        }
        __syncthreads();
        const I2 c = lidCell(w, wid);
        const uint32_t h = heldAt(w, c);
        if (h != NONE) atomicMin(&first, h);
        __syncthreads();
        const uint32_t f0 = first;
        if (h != NONE) {
            int32_t d[3];
            heldPush(w, c, h, d);
            if ((D.blocks[w.stateSlot(w.blockIndex(w.activeBlock(wid)))] & NEAR_LIQUID) != 0u)
                atomicOr(&D.motion[liquidSlot(h, 3u)], WIG_LIQUID_WET);
            for (uint32_t k = 0; k < 3; k++) {
                if (h == f0) atomicAdd(&sums[k], (uint32_t)d[k]);
                else atomicAdd(&D.motion[liquidSlot(h, k)], (uint32_t)d[k]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && f0 != NONE)
            for (uint32_t k = 0; k < 3; k++) atomicAdd(&D.motion[liquidSlot(f0, k)], sums[k]);
        __syncthreads();
    }
}

// bodyPush (fluid.wgsl:3205-3218): a thread a body.
__global__ void k_bodyPush(Dev D) {
    W w(D);
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= MAX_BODIES) return;
    const V3 ch = add3(add3(pushChangeFree(w, b, PUSH_SURFACE), pushChangeFree(w, b, PUSH_DRAG)), pushChangeFree(w, b, PUSH_F));
    if (ch.x == 0.0f && ch.y == 0.0f && ch.z == 0.0f) return;
    atomicAdd(&D.motion[liquidSlot(b, 0u)], (uint32_t)f2i(rnd_even(ch.x * WIG_RIGID_FIX)));
    atomicAdd(&D.motion[liquidSlot(b, 1u)], (uint32_t)f2i(rnd_even(ch.y * WIG_RIGID_FIX)));
    atomicAdd(&D.motion[liquidSlot(b, 2u)], (uint32_t)f2i(rnd_even(ch.z * WIG_RIGID_FIX)));
}

static inline unsigned block_grid(const Dev& D, unsigned per_sm) {
    unsigned g = 148u * per_sm;
    return D.B < g ? (D.B ? D.B : 1u) : g;
}

unsigned list_grid(const BatchShape& S, uint32_t list, unsigned per_sm) {
    const unsigned g = 148u * per_sm, n = S.max_items[list];
    return n < g ? (n ? n : 1u) : g;
}

int launch_pass(const Batch& Bt, const BatchShape& S, const Dev& D0, int pass, uint32_t level, uint32_t cycle,
                cudaStream_t s) {
    // the passes shared by every form: over the batch's work lists
    const unsigned A = list_grid(S, L_ACT, 32), WB = list_grid(S, L_WB, 32);
    const unsigned PS = list_grid(S, L_PS, 8), PP = list_grid(S, L_PP, 8);
    const unsigned RET = list_grid(S, L_RET, 32), ONE = list_grid(S, L_ONE, 2), ALL = list_grid(S, L_ONE_ALL, 2);
    // the plain form's solve: world 0 alone
    const unsigned G = block_grid(D0, 32);
    auto lvl = [&](uint32_t l) {
        return dim3((D0.level_w[l] + 7u) / 8u, (D0.level_h[l] + 7u) / 8u);
    };
    const Dev& D = D0;
    switch (pass) {
    case WIG_PASS_SYNC: k_sync<<<WB, 64, 0, s>>>(Bt, 1); break;
    case WIG_PASS_SYNC_MARKS: k_sync<<<WB, 64, 0, s>>>(Bt, 0); break;
    case WIG_PASS_SYNC_PARTICLES: k_syncParticles<<<PS, 256, 0, s>>>(Bt); break;
    case WIG_PASS_SYNC_SEED: k_syncSeed<<<WB, 64, 0, s>>>(Bt); break;
    case WIG_PASS_COMPACT: k_compact<<<ALL, 1024, 0, s>>>(Bt); break;
    case WIG_PASS_RETIRE: k_retire<<<RET, 64, 0, s>>>(Bt); break;
    case WIG_PASS_CLEAR: k_clear<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_GATHER: k_gather<<<PP, 256, 0, s>>>(Bt); break;
    case WIG_PASS_SEAL_JOIN: k_sealJoin<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_SEAL_ANCHOR: k_sealAnchor<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_CLASSIFY: k_classify<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_SET_FACES: k_setFaces<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_VISCOSITY_RED: k_viscosity<<<A, 64, 0, s>>>(Bt, 0); break;
    case WIG_PASS_VISCOSITY_BLACK: k_viscosity<<<A, 64, 0, s>>>(Bt, 1); break;
    case WIG_PASS_UNPRESS: k_viscosity<<<A, 64, 0, s>>>(Bt, 2); break;
    case WIG_PASS_DIVERGENCE: k_divergence<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_CG_START: k_cgStart<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_CG_JOIN: k_cgJoin<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_CG_ANCHOR: k_cgAnchor<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_CG_RESIDUAL: k_cgResidual<<<G, 64, 0, s>>>(D); break;
    case WIG_PASS_CG_PREPARE: k_cgPrepare<<<G, 64, 0, s>>>(D); break;
    case WIG_PASS_RELAX_RIMS: k_relaxRims<<<G, 64, 0, s>>>(D, cycle); break;
    case WIG_PASS_RELAX: k_relax<<<G, 64, 0, s>>>(D, 0, cycle); break;
    case WIG_PASS_RELAX_SHIFTED: k_relax<<<G, 64, 0, s>>>(D, BLOCK / 2, cycle); break;
    case WIG_PASS_RESTRICT: k_restrict<<<lvl(level), dim3(8, 8), 0, s>>>(D, level, cycle); break;
    case WIG_PASS_SMOOTH_RED: k_smooth<<<lvl(level), dim3(8, 8), 0, s>>>(D, level, 0, cycle); break;
    case WIG_PASS_SMOOTH_BLACK: k_smooth<<<lvl(level), dim3(8, 8), 0, s>>>(D, level, 1, cycle); break;
    case WIG_PASS_SOLVE: k_solve<<<1, 512, 0, s>>>(D, level, cycle); break;
    case WIG_PASS_PROLONG: k_prolong<<<lvl(level), dim3(8, 8), 0, s>>>(D, level, cycle); break;
    case WIG_PASS_PROLONG_FINE: k_prolongFine<<<G, 64, 0, s>>>(D, cycle); break;
    case WIG_PASS_CG_RHO: k_cgRho<<<G, 64, 0, s>>>(D, cycle); break;
    case WIG_PASS_CG_BETA: k_cgBeta<<<1, 256, 0, s>>>(D, cycle); break;
    case WIG_PASS_CG_DIRECTION: k_cgDirection<<<G, 64, 0, s>>>(D, cycle); break;
    case WIG_PASS_CG_APPLY: k_cgApply<<<G, 64, 0, s>>>(D, cycle); break;
    case WIG_PASS_CG_ALPHA: k_cgAlpha<<<1, 256, 0, s>>>(D, cycle); break;
    case WIG_PASS_CG_UPDATE: k_cgUpdate<<<G, 64, 0, s>>>(D, cycle); break;
    case WIG_PASS_CG_FINISH: k_cgFinish<<<G, 64, 0, s>>>(D); break;
    case WIG_PASS_PROJECT: k_project<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_EXTRAPOLATE: k_extrapolate<<<A, 64, 0, s>>>(Bt, 1u); break;
    case WIG_PASS_EXTRAPOLATE_FURTHER: k_extrapolate<<<A, 64, 0, s>>>(Bt, 2u); break;
    case WIG_PASS_ADVECT: k_advect<<<PP, 256, 0, s>>>(Bt); break;
    case WIG_PASS_SORT_COUNT: k_sortCount<<<PP, 256, 0, s>>>(Bt); break;
    case WIG_PASS_SCAN_BLOCKS: k_scanBlocks<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_SCAN_TOTALS: k_scanTotals<<<ONE, 256, 0, s>>>(Bt); break;
    case WIG_PASS_SCAN_FINISH: k_scanFinish<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_SCATTER: k_scatter<<<PP, 256, 0, s>>>(Bt); break;
    case WIG_PASS_RASTER_CLAIMS: k_rasterClaims<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_RASTER: k_raster<<<A, 64, 0, s>>>(Bt); break;
    case WIG_PASS_UNPAINT: k_unpaint<<<A, 64, 0, s>>>(Bt); break;
    default:
        // the bodies' passes: world 0 with its bodies bound (no-ops without)
        if (pass < WIG_PASS_BODY_START || pass > WIG_PASS_BODY_PUSH) return WIG_E_ARG;
        if (!D.motion || !D.pushes) return WIG_OK;
        switch (pass) {
        case WIG_PASS_BODY_START: k_bodyStart<<<(MAX_BODIES * WIG_BODY_PUSH_WORDS + 255u) / 256u, 256, 0, s>>>(D); break;
        case WIG_PASS_BODY_LOADS: k_bodyLoads<<<G, 64, 0, s>>>(D); break;
        case WIG_PASS_BODY_DRAG: k_bodyDrag<<<G, 64, 0, s>>>(D); break;
        case WIG_PASS_BODY_FACES: k_bodyFaces<<<G, 64, 0, s>>>(D); break;
        case WIG_PASS_CG_BODY_X: k_cgBody<<<G, 64, 0, s>>>(D, 0, cycle); break;
        case WIG_PASS_CG_BODY_P: k_cgBody<<<G, 64, 0, s>>>(D, 1, cycle); break;
        case WIG_PASS_CG_BODY_F: k_cgBody<<<G, 64, 0, s>>>(D, 2, cycle); break;
        case WIG_PASS_RIGIDIFY: k_rigidify<<<G, 64, 0, s>>>(D); break;
        case WIG_PASS_BODY_PUSH: k_bodyPush<<<(MAX_BODIES + 255u) / 256u, 256, 0, s>>>(D); break;
        default: break;
        }
        break;
    }
    return WIG_OK;
}

void launch_labels(const Batch& Bt, const BatchShape& S, cudaStream_t s, int part) {
    const unsigned A = list_grid(S, L_ACT, 32);
    if (part == 0) k_cgStartLocal<<<A, 64, 0, s>>>(Bt);
    else k_cgJoinAcross<<<A, 64, 0, s>>>(Bt);
}

int launch_norm(const Dev& D, int which, uint32_t cycle, cudaStream_t s) {
    k_norm<<<1, 256, 0, s>>>(D, which, cycle);
    return WIG_OK;
}

}  // namespace wig
