// wig_fast.cu — the fast form of the liquid's pressure solve (the CG loop
// of encodeFluid, js/sim.js:2551-2591; fluid.wgsl:2047-2893).
//
// Same arithmetic as the reference's passes, operation for operation and in
// the same order (so every value the step leaves is bit-for-bit the plain
// form's), arranged for the GPU:
//   * the stencil's coefficients (fineBeta on the cells, faceBeta on the
//     coarse levels) are worked out once a step and kept, instead of being
//     recomputed with their divisions in every sweep;
//   * the vectors live in structure-of-arrays scratch (a float per cell,
//     row-major), so a warp's loads are contiguous instead of 32-44 bytes
//     apart as in the reference's per-cell records;
//   * the levels of at most 4096 cells, down to the coarsest and back, are
//     one CTA's work in shared memory, one launch instead of ~15;
//   * the CG's block sums finish in the last block to write its partial (a
//     threadfence reduction: the same fixed tree order, one launch fewer);
//   * the iterations are the body of a CUDA-graph WHILE node: a step runs as
//     many as it needs, with no launches for the converged ones.
// The scratch keeps one invariant: level-0 arrays are zero outside the
// blocks worked on (zeroed at allocation, when a world is uploaded, and as
// blocks retire), where the reference's field is zero too.

#include <algorithm>

#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include "wig_fast.cuh"

namespace wig {
namespace {

__device__ __forceinline__ uint32_t vld(const uint32_t* p) { return *(const volatile uint32_t*)p; }
__device__ __forceinline__ double vldd(const double* p) { return *(const volatile double*)p; }
__device__ __forceinline__ float vldf(const float* p) { return *(const volatile float*)p; }

__device__ __forceinline__ I2 lidCell(const W& w, uint32_t wid) {
    I2 b = w.activeBlock(wid);
    return I2{b.x * BLOCK + (int)(threadIdx.x & 7u), b.y * BLOCK + (int)(threadIdx.x >> 3)};
}

// Neighbour d (left, right, up, down: beside, fluid.wgsl:267-269) of cell
// (x, y) on a w x h level, clamped onto the cell itself past the edge (its
// coefficient there is 0).
__device__ __forceinline__ uint32_t nbr(uint32_t i, int x, int y, int w, int h, int d) {
    switch (d) {
    case 0: return x > 0 ? i - 1u : i;
    case 1: return x < w - 1 ? i + 1u : i;
    case 2: return y > 0 ? i - (uint32_t)w : i;
    default: return y < h - 1 ? i + (uint32_t)w : i;
    }
}
__device__ __forceinline__ bool nbrIn(int x, int y, int w, int h, int d) {
    switch (d) {
    case 0: return x > 0;
    case 1: return x < w - 1;
    case 2: return y > 0;
    default: return y < h - 1;
    }
}

// A 256-thread CTA's four trees of 64 (sumBlock's, fluid.wgsl:2628-2641),
// one per tile of 64 threads; each tile's sum for all its threads.
template <class T>
__device__ __forceinline__ T tree64x4(T* s, T v) {
    const int lane = (int)(threadIdx.x & 63u), base = (int)(threadIdx.x & ~63u);
    s[threadIdx.x] = v;
    __syncthreads();
    for (int h = 32; h > 0; h >>= 1) {
        if (lane < h) s[base + lane] = s[base + lane] + s[base + lane + h];
        __syncthreads();
    }
    T r = s[base];
    __syncthreads();
    return r;
}

// The same trees of 64 in two halves, one barrier between them: tilePut,
// in the upper warp of each tile, leaves its 32 values in s (128 entries);
// after a barrier, tileSum, in the lower warp, adds them (the tree's first
// step, lane + 32) and finishes the tree by shuffles (lane + h, h = 16 ..
// 1): the same additions in the same order.  The tile's sum is in its
// thread 0.  A kernel alternates two buffers between items, so one item's
// sums and the next item's puts never share one.
template <class T>
__device__ __forceinline__ void tilePut(T* s, T v) {
    const uint32_t lane = threadIdx.x & 63u;
    if (lane >= 32u) s[((threadIdx.x >> 6) << 5) + (lane - 32u)] = v;
}
template <class T>
__device__ __forceinline__ T tileSum(const T* s, T v) {
    if ((threadIdx.x & 32u) == 0u) {  // a whole warp: the tile's lower
        v = v + s[((threadIdx.x >> 6) << 5) + (threadIdx.x & 31u)];
#pragma unroll
        for (int h = 16; h > 0; h >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, h);
    }
    return v;
}

// sumBlocks (fluid.wgsl:2645-2661) by a 256-thread CTA, component comp of 2
// of the active blocks' partials: thread li adds the partials of blocks li,
// li + 256, ... in that order (loaded ahead in coalesced batches of 16, the
// adds kept in order), then the tree over the 256.
template <class T>
__device__ T sumBlocks256(const W& w, const T* part, int comp, T* s) {
    const uint32_t B = w.D.B;
    const uint32_t* state = w.D.blocks + B;
    const uint32_t li = threadIdx.x;
    T acc = T(0);
    for (uint32_t k0 = li; k0 < B; k0 += 256u * 16u) {
        T v[16];
        uint32_t st[16];
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const uint32_t k = k0 + 256u * (uint32_t)u;
            st[u] = k < B ? __ldcg(&state[k]) : 0u;
            v[u] = k < B ? __ldcg(&part[2u * k + (uint32_t)comp]) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 16; u++)
            if ((st[u] & ACTIVE) != 0u) acc = acc + v[u];
    }
    s[li] = acc;
    __syncthreads();
    for (int h = 128; h > 32; h >>= 1) {
        if ((int)li < h) s[li] = s[li] + s[li + h];
        __syncthreads();
    }
    if (li < 32u) {
        T v = s[li] + s[li + 32u];
#pragma unroll
        for (int h = 16; h > 0; h >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, h);
        if (li == 0u) s[0] = v;
    }
    __syncthreads();
    T r = s[0];
    __syncthreads();
    return r;
}

// sumBlocks of both components of the partials in one pass (each component
// in sumBlocks256's order).
template <class T>
__device__ void sumBlocks256x2(const W& w, const T* part, T* s0, T* s1, T* out0, T* out1) {
    const uint32_t B = w.D.B;
    const uint32_t* state = w.D.blocks + B;
    const uint32_t li = threadIdx.x;
    T a0 = T(0), a1 = T(0);
    for (uint32_t k0 = li; k0 < B; k0 += 256u * 16u) {
        T v0[16], v1[16];
        uint32_t st[16];
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const uint32_t k = k0 + 256u * (uint32_t)u;
            st[u] = k < B ? __ldcg(&state[k]) : 0u;
            v0[u] = k < B ? __ldcg(&part[2u * k]) : T(0);
            v1[u] = k < B ? __ldcg(&part[2u * k + 1u]) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 16; u++)
            if ((st[u] & ACTIVE) != 0u) {
                a0 = a0 + v0[u];
                a1 = a1 + v1[u];
            }
    }
    s0[li] = a0;
    s1[li] = a1;
    __syncthreads();
    for (int h = 128; h > 32; h >>= 1) {
        if ((int)li < h) {
            s0[li] = s0[li] + s0[li + h];
            s1[li] = s1[li] + s1[li + h];
        }
        __syncthreads();
    }
    if (li < 32u) {
        T v0 = s0[li] + s0[li + 32u], v1 = s1[li] + s1[li + 32u];
#pragma unroll
        for (int h = 16; h > 0; h >>= 1) {
            v0 = v0 + __shfl_down_sync(0xffffffffu, v0, h);
            v1 = v1 + __shfl_down_sync(0xffffffffu, v1, h);
        }
        if (li == 0u) {
            s0[0] = v0;
            s1[0] = v1;
        }
    }
    __syncthreads();
    *out0 = s0[0];
    *out1 = s1[0];
    __syncthreads();
}

// Whether this CTA counted the last of `total` tiles: a threadfence
// reduction's test.  The partials of the counted tiles were written by the
// tiles' first threads (threadIdx.x % 64 == 0), each with no fence of its
// own: those threads fence here, once for all the tiles of the run, before
// the count.
__device__ bool lastOf4(uint32_t* counter, uint32_t inc, uint32_t total) {
    __shared__ int last;
    if ((threadIdx.x & 63u) == 0u) __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t old = atomicAdd(counter, inc);
        last = old + inc == total ? 1 : 0;
        if (last) {
            *counter = 0u;
            __threadfence();
        }
    }
    __syncthreads();
    return last != 0;
}

// Whether a CTA's run over a list ends its share of a world at item g (the
// run's last item, or the next item is another world's): where it counts
// the tiles it finished, one atomic per world a CTA instead of one per item.
__device__ __forceinline__ bool worldRunEnds(const Batch& Bt, uint32_t list, uint32_t g, uint32_t e, uint32_t it) {
    if (g + 1u >= e) return true;
    return ((uint64_t)Bt.item(list, g + 1u) >> Bt.lbits) != ((uint64_t)it >> Bt.lbits);
}

// At the end of a world's run: counts the CTA's pending tiles of that world;
// true in the CTA that counted the world's last tile.
__device__ __forceinline__ bool flushTiles(const Batch& Bt, uint32_t g, uint32_t e, uint32_t it, uint32_t& pend,
                                           uint32_t* counter, uint32_t total) {
    if (!worldRunEnds(Bt, L_ACT4, g, e, it)) return false;
    const uint32_t inc = pend;
    pend = 0u;
    return lastOf4(counter, inc, total);
}

__device__ __forceinline__ I2 tileCell(const W& w, uint32_t wid) {
    I2 b = w.activeBlock(wid);
    return I2{b.x * BLOCK + (int)(threadIdx.x & 7u), b.y * BLOCK + (int)((threadIdx.x >> 3) & 7u)};
}

// Where a kernel finds its items' world: in a batch of one, the world
// itself, a kernel parameter (read as constants, with no load at a CTA's
// start); else the CTA's shared copy of the world-table entry.
template <bool ONE>
struct WorldSrc;
template <>
struct WorldSrc<true> {
    World w;
    __device__ __forceinline__ const World& get(const Batch&, uint32_t, WorldCopy&) const { return w; }
    __device__ __forceinline__ const World& getG(const Batch&, uint32_t) const { return w; }
};
template <>
struct WorldSrc<false> {
    __device__ __forceinline__ const World& get(const Batch& Bt, uint32_t it, WorldCopy& c) const {
        return worldOf(Bt, it, c);
    }
    // without the CTA's copy (a warp's own item)
    __device__ __forceinline__ const World& getG(const Batch& Bt, uint32_t it) const { return Bt.world(it); }
};

// An item's world: its descriptor D, fast scratch F, accessors w, unit j,
// from the CTA's copy of the world (every thread of the CTA, each item in
// turn; the kernel declares `__shared__ WorldCopy wc_;`) or (FAST_ITEM_G)
// from the world table.
#define FAST_ITEM(Bt, it, D, F, w, j)            \
    const World& Wd_##it = src.get((Bt), (it), wc_); \
    const Dev& D = Wd_##it.D;                    \
    const FastW& F = Wd_##it.S;                  \
    const W w(D);                                \
    const uint32_t j = (Bt).unit(it)
#define FAST_ITEM_G(Bt, it, D, F, w, j)          \
    const World& Wd_##it = (Bt).world(it);       \
    const Dev& D = Wd_##it.D;                    \
    const FastW& F = Wd_##it.S;                  \
    const W w(D);                                \
    const uint32_t j = (Bt).unit(it)

// ================================================================ set-up

// cgStart, cgResidual, cgPrepare (fluid.wgsl:2665-2732) into the scratch,
// the cells' coefficients worked out (four tiles a 256-thread CTA, a world's
// group of four active blocks an item; the CTA that counts a world's last
// tile sums its ||b||^2), and the blocks that dropped out this step zeroed
// (the invariant).
template <bool ONE>
__global__ void __launch_bounds__(256) k_fSetup(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    __shared__ double s64[256];
    uint32_t pend_ = 0;  // tiles finished of the current world, not yet counted
    FOR_ITEMS(Bt, L_ACT4, it) {
        FAST_ITEM(Bt, it, D, F, w, g);
        const uint32_t na = w.activeCount();
        const bool tol = D.st->tol_mode != 0u;
        const Lvl& L0 = F.L[0];
        const uint32_t wid = g * 4u + (threadIdx.x >> 6);
        const bool valid = wid < na;
        double b2 = 0.0;
        I2 c{-1, -1};
        if (valid) c = tileCell(w, wid);
        if (valid && w.inWorld(c)) {
            const uint32_t i = w.cellIndex(c);
            const float4 gc = w.f4(2u * i), dr = w.f4(2u * i + 1u);
            const float rho = gc.z;
            L0.rho[i] = rho;
            F.X[i] = gc.x;
            F.P[i] = 0.0f;
            F.Q[i] = 0.0f;
            L0.px[i] = 0.0f;
            L0.py[i] = dr.x;
            L0.ry[i] = dr.y;
            F.rimx[i] = 0.0f;
            F.rimy[i] = dr.x;
            float bb[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            float R = 0.0f, pinv = 0.0f;
            uint8_t mask = 0;
            if (rho > 0.0f) {
                const float share = w.densityAt(c);
                float sx = 0.0f, dg = 0.0f;
                for (int d = 0; d < 4; d++) {
                    I2 n = beside(c, d);
                    if (!w.inWorld(n)) continue;
                    float4 gn = w.f4(2u * w.cellIndex(n));
                    float r = gn.z;
                    if (r < 0.0f) continue;
                    float beta = fineBeta(rho, r, share, w.densityAt(n));
                    bb[d] = beta;
                    if (r > 0.0f) mask |= (uint8_t)(1u << d);
                    // the stencil over the warm pressure (cgResidual runs before cgPrepare)
                    sx = sx + beta * gn.x;
                    dg = dg + beta;
                }
                pinv = (vld(w.gwp(i, G_REGION)) == i) ? PIN : 0.0f;
                float res = gc.y - (sx - (dg + pinv) * gc.x) / 1.0f;
                R = -res - 0.0f;
                double bd = (double)gc.y;
                b2 = bd * bd;
            }
            L0.b0[i] = bb[0]; L0.b1[i] = bb[1]; L0.b2[i] = bb[2]; L0.b3[i] = bb[3];
            L0.diag[i] = bb[0] + bb[1] + bb[2] + bb[3];
            if (Bt.mixed) {
                // the smoother's copies of the coefficients (the mixed form)
                __half* h = F.H[0].base;
                const uint32_t n = F.H[0].n;
                h[i] = __float2half_rn(bb[0]);
                h[n + i] = __float2half_rn(bb[1]);
                h[2u * n + i] = __float2half_rn(bb[2]);
                h[3u * n + i] = __float2half_rn(bb[3]);
            }
            F.pin[i] = pinv;
            F.fmask[i] = mask;
            F.R[i] = R;
            L0.rx[i] = rho > 0.0f ? -R : 0.0f;
        }
        if (tol) {
            double v = tree64x4(s64, b2);
            if (valid && (threadIdx.x & 63u) == 0u) {
                D.norm64[2u * w.blockIndex(w.activeBlock(wid))] = v;
            }
            pend_ += min(4u, na - g * 4u);
            if (flushTiles(Bt, g_it, e_it, it, pend_, &D.st->fdone[0], na)) {
                double bn = sumBlocks256(w, D.norm64, 0, s64);
                if (threadIdx.x == 0) {
                    D.st->bnorm2 = bn;
                    D.st->rel = 1.0;
                }
            }
        }
    }
    // the blocks that dropped out: their level-0 arrays back to zero (a
    // retired block a quarter of the CTA)
    const uint32_t nr = Bt.n(L_RET);
    for (uint32_t t = blockIdx.x * 4u + (threadIdx.x >> 6); t < nr; t += gridDim.x * 4u) {
        const uint32_t it = Bt.item(L_RET, t);
        FAST_ITEM_G(Bt, it, D, F, w, j);
        uint32_t n = D.blocks[w.retiredSlot(j)];
        const I2 bq_ = w.blockAt(n);
        I2 c{bq_.x * BLOCK + (int)(threadIdx.x & 7u), bq_.y * BLOCK + (int)((threadIdx.x >> 3) & 7u)};
        if (w.inWorld(c)) {
            uint32_t i = w.cellIndex(c);
            const Lvl& L0 = F.L[0];
            L0.px[i] = 0.0f; L0.py[i] = 0.0f; L0.rho[i] = 0.0f;
            F.rimx[i] = 0.0f; F.rimy[i] = 0.0f; F.P[i] = 0.0f;
        }
    }
}

// The level-0 arrays neighbours read, zeroed in the blocks not worked on
// (the invariant), for worlds whose scratch is lent by a pool for the step:
// a CTA per block of the world.
__global__ void k_fZeroIdle(Batch Bt) {
    FOR_ITEMS(Bt, L_WB, it) {
        FAST_ITEM_G(Bt, it, D, F, w, n);
        if (D.st->book != 0u || (D.blocks[w.stateSlot(n)] & ACTIVE) != 0u) continue;
        for (uint32_t t = threadIdx.x; t < 64u; t += blockDim.x) {
            const I2 bq_ = w.blockAt(n);
            I2 c{bq_.x * BLOCK + (int)(t & 7u), bq_.y * BLOCK + (int)(t >> 3)};
            if (!w.inWorld(c)) continue;
            const uint32_t i = w.cellIndex(c);
            F.L[0].px[i] = 0.0f; F.L[0].py[i] = 0.0f; F.L[0].rho[i] = 0.0f;
            F.rimx[i] = 0.0f; F.rimy[i] = 0.0f; F.P[i] = 0.0f;
        }
    }
}

// Zeroes the level-0 arrays the neighbours read (after an upload).
__global__ void k_fZero(FastW F, uint32_t C) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
        F.L[0].px[i] = 0.0f; F.L[0].py[i] = 0.0f; F.L[0].rho[i] = 0.0f;
        F.rimx[i] = 0.0f; F.rimy[i] = 0.0f; F.P[i] = 0.0f;
    }
}

// ================================================================ level storage

// A level's arrays as stored, the operator (density, stencil coefficients,
// diagonal) in T: f32 (the plain precision) or binary16 (the mixed form);
// values are read into and worked in f32.  The potentials, right-hand sides and way-up potentials of a level whose
// operator is stored as T: f32 with an f32 operator; bf16 (8 bits of
// mantissa, f32's range, so no scaling as a residual shrinks) with the mixed
// form's binary16 operator.  Both are stored in the level's f32 arrays (a
// bf16 array fills the first half of one).
template <class T>
struct PotOf {
    using type = float;
};
template <>
struct PotOf<__half> {
    using type = __nv_bfloat16;
};
// A level's arrays: potentials and right-hand sides of P, densities of R,
// the stencil's coefficients (and, when B is f32, their stored sum) of B.
template <class P, class R, class B>
struct LRefX {
    P *px, *py, *rx, *ry;
    R* rho;
    B *b0, *b1, *b2, *b3, *diag;
};
// Levels 1 down as the form stores them (operator T).
template <class T>
using LRef = LRefX<typename PotOf<T>::type, T, T>;
// Level 0 as the form's smoother reads it: all f32, or (the mixed form) its
// coefficients from their binary16 copies, the potentials, right-hand sides
// and densities f32 (the CG's A p keeps the f32 coefficients).
template <class T>
using L0Ref = LRefX<float, float, T>;
__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __half* p) { return __half2float(*p); }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void st(float* p, float v) { *p = v; }
__device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
__device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

template <class T>
__device__ __forceinline__ LRef<T> lref(const FastW& F, uint32_t l);
template <>
__device__ __forceinline__ LRef<float> lref<float>(const FastW& F, uint32_t l) {
    const Lvl& V = F.L[l];
    return LRef<float>{V.px, V.py, V.rx, V.ry, V.rho, V.b0, V.b1, V.b2, V.b3, V.diag};
}
template <>
__device__ __forceinline__ LRef<__half> lref<__half>(const FastW& F, uint32_t l) {
    const Lvl& V = F.L[l];
    __half* b = F.H[l].base;
    const uint32_t n = F.H[l].n;
    using P = __nv_bfloat16;
    return LRef<__half>{reinterpret_cast<P*>(V.px), reinterpret_cast<P*>(V.py), reinterpret_cast<P*>(V.rx),
                        reinterpret_cast<P*>(V.ry), b, b + n, b + 2u * n, b + 3u * n, b + 4u * n, nullptr};
}
template <class T>
__device__ __forceinline__ L0Ref<T> lref0(const FastW& F);
template <>
__device__ __forceinline__ L0Ref<float> lref0<float>(const FastW& F) {
    return lref<float>(F, 0u);
}
template <>
__device__ __forceinline__ L0Ref<__half> lref0<__half>(const FastW& F) {
    const Lvl& V = F.L[0];
    __half* b = F.H[0].base;
    const uint32_t n = F.H[0].n;
    return L0Ref<__half>{V.px, V.py, V.rx, V.ry, V.rho, b, b + n, b + 2u * n, b + 3u * n, nullptr};
}
// Level l's way-up potentials (l >= 1) as a level of operator T stores them.
template <class T>
__device__ __forceinline__ typename PotOf<T>::type* upx(const FastW& F, uint32_t l) {
    return reinterpret_cast<typename PotOf<T>::type*>(F.L[l].ux);
}
template <class T>
__device__ __forceinline__ typename PotOf<T>::type* upy(const FastW& F, uint32_t l) {
    return reinterpret_cast<typename PotOf<T>::type*>(F.L[l].uy);
}

// A cell's diagonal: stored in f32 (the sum of its four coefficients, in
// that order); in binary16 not stored but the sum of the rounded
// coefficients, so the rounded operator keeps its diagonal equal to the sum
// of its off-diagonals (a separately rounded diagonal could fall below it
// and make a region with no free surface indefinite).
template <class P, class R>
__device__ __forceinline__ float diagAt(const LRefX<P, R, float>& V, uint32_t k) { return V.diag[k]; }
template <class P, class R>
__device__ __forceinline__ float diagAt(const LRefX<P, R, __half>& V, uint32_t k) {
    return ((ld(V.b0 + k) + ld(V.b1 + k)) + ld(V.b2 + k)) + ld(V.b3 + k);
}

// ================================================================ relaxation

__device__ I2 tileBlockF(const W& w, uint32_t wid, int shift) {
    if (wid < w.activeCount()) return w.activeBlock(wid);
    int wide = (int)w.D.BW, high = (int)w.D.BH;
    int j = (int)wid - (int)w.D.B;
    if (shift == 0 || j < 0 || j > high + wide) return I2{-1, -1};
    return j <= high ? I2{wide, j} : I2{j - high - 1, high};
}

// relaxTile (fluid.wgsl:2109-2182) over the scratch: the rim snapshot's
// values for liquid cells, the potentials (zero) elsewhere.  A warp a tile
// (four a CTA, each warp its own run of the list): lane l holds the red and
// the black cell of quarter l % 4 of row l / 4, so every lane works in every
// sweep and a sweep ends at a warp barrier.  Within a colour the cells are
// independent, so each keeps the reference's arithmetic and order.
// `second`: the iteration's relaxation after the V-cycle, on the other
// tiling from the first (each world's first tiling is its step's).
template <bool ONE, class T>
__global__ void __launch_bounds__(128) k_fRelax(Batch Bt, const __grid_constant__ WorldSrc<ONE> src, int second) {
    __shared__ float tpx[4][RIM * RIM], tpy[4][RIM * RIM];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    float* sx_ = tpx[warp];
    float* sy_ = tpy[warp];
    const uint32_t n = Bt.n(L_RELAX);
    const uint32_t warps = gridDim.x * 4u, per = (n + warps - 1u) / warps;
    const uint32_t first = (blockIdx.x * 4u + warp) * per, last = min(first + per, n);
    for (uint32_t g = first; g < last; g++) {
        const uint32_t it = Bt.item(L_RELAX, g);
        const World& Wd = src.getG(Bt, it);
        const Dev& D = Wd.D;
        const FastW& F = Wd.S;
        const W w(D);
        const uint32_t j = Bt.unit(it);
        if (D.st->cont == 0u) continue;
        const int shift = ((D.st->shift_first ^ (uint32_t)second) & 1u) ? BLOCK / 2 : 0;
        const Lvl& L0 = F.L[0];
        const uint32_t na = w.activeCount();
        const uint32_t wid = j < na ? j : D.B + (j - na);
        const I2 b = tileBlockF(w, wid, shift);
        const int ox = b.x * BLOCK - shift, oy = b.y * BLOCK - shift;
        if (b.x < 0 || ox >= D.W || oy >= D.H) continue;
        if ((w.statesOf(I2{ox / BLOCK, oy / BLOCK}, I2{(ox + BLOCK - 1) / BLOCK, (oy + BLOCK - 1) / BLOCK}) & HAS_FLUID) == 0u)
            continue;
        // the lane's two cells first (independent of the tile's loads)
        const int ly = (int)(lane >> 2), q = (int)(lane & 3u);
        const int p0 = (ox + oy + ly) & 1;
        int t[2];
        uint32_t idx[2];
        bool solving[2], visc[2];
        float rx[2], ry[2], bx[2], by[2], bz[2], bw[2], dxx[2], dyy[2];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int lx = 2 * q + (c == 0 ? p0 : 1 - p0);
            const I2 me{ox + lx, oy + ly};
            t[c] = (ly + 1) * RIM + lx + 1;
            float r_x = 0.0f, r_y = 0.0f, b0 = 0.0f, b1 = 0.0f, b2 = 0.0f, b3 = 0.0f, dg = 0.0f, pv = 0.0f;
            uint32_t id = 0;
            bool fluid = false;
            if (w.inWorld(me)) {
                id = w.cellIndex(me);
                const L0Ref<T> S0 = lref0<T>(F);
                fluid = L0.rho[id] > 0.0f;
                r_x = L0.rx[id];
                r_y = L0.ry[id];
                b0 = ld(S0.b0 + id);
                b1 = ld(S0.b1 + id);
                b2 = ld(S0.b2 + id);
                b3 = ld(S0.b3 + id);
                dg = diagAt(S0, id);
                pv = F.pin[id];
            }
            if (!fluid) {
                r_x = 0.0f; r_y = 0.0f; b0 = 0.0f; b1 = 0.0f; b2 = 0.0f; b3 = 0.0f; dg = 0.0f; pv = 0.0f;
            }
            idx[c] = id;
            rx[c] = r_x; ry[c] = r_y; bx[c] = b0; by[c] = b1; bz[c] = b2; bw[c] = b3;
            dxx[c] = dg + pv;
            dyy[c] = fmaxf(dg, 1e-30f);
            solving[c] = fluid && dxx[c] > 0.0f;
            visc[c] = dg > 0.0f;
        }
        // the tile and its rim: the snapshot's values for liquid cells, the
        // potentials elsewhere
        // (the four rounds of the lane's loads issued together)
        {
            constexpr int NR = (RIM * RIM + 31) / 32;
            float rr[NR], ax[NR], ay[NR], qx[NR], qy[NR];
            bool inw[NR];
#pragma unroll
            for (int u = 0; u < NR; u++) {
                const int k = (int)lane + 32 * u;
                const I2 c{ox - 1 + k % RIM, oy - 1 + k / RIM};
                inw[u] = k < RIM * RIM && w.inWorld(c);
                const uint32_t i = inw[u] ? w.cellIndex(c) : 0u;
                rr[u] = L0.rho[i];
                ax[u] = F.rimx[i];
                ay[u] = F.rimy[i];
                qx[u] = L0.px[i];
                qy[u] = L0.py[i];
            }
#pragma unroll
            for (int u = 0; u < NR; u++) {
                const int k = (int)lane + 32 * u;
                if (k >= RIM * RIM) continue;
                float px = 0.0f, py = 0.0f;
                if (inw[u]) {
                    px = rr[u] > 0.0f ? ax[u] : qx[u];
                    py = rr[u] > 0.0f ? ay[u] : qy[u];
                }
                sx_[k] = px;
                sy_[k] = py;
            }
        }
        __syncwarp();
        for (int sw = 0; sw < 2 * SWEEPS; sw++) {
            const int c = sw & 1;
            if (solving[c]) {
                const int tc = t[c];
                float sx = bx[c] * sx_[tc - 1] + by[c] * sx_[tc + 1] + bz[c] * sx_[tc - RIM] + bw[c] * sx_[tc + RIM];
                float sy = bx[c] * sy_[tc - 1] + by[c] * sy_[tc + 1] + bz[c] * sy_[tc - RIM] + bw[c] * sy_[tc + RIM];
                float nx = mixf(sx_[tc], (sx - rx[c]) / dxx[c], SMOOTH_OMEGA);
                float ny = mixf(sy_[tc], (sy - ry[c]) / dyy[c], SMOOTH_OMEGA);
                sx_[tc] = nx;
                if (visc[c]) sy_[tc] = ny;
            }
            __syncwarp();
        }
#pragma unroll
        for (int c = 0; c < 2; c++)
            if (solving[c]) {
                L0.px[idx[c]] = sx_[t[c]];
                L0.py[idx[c]] = sy_[t[c]];
            }
        __syncwarp();
    }
}

// ================================================================ the levels

// residualAt (fluid.wgsl:2306-2315) of cell k on a level held in arrays with
// stored coefficients (level 0's pinned roots held at PIN).  The division by
// h2, a power of two, is the multiplication by its exact inverse: the same
// real number rounded once either way, so the same bits.
template <class VT>
__device__ __forceinline__ V2 residualStored(const VT& V, const float* pin, uint32_t k, int x, int y, int lw, int lh,
                                             float inv_h2) {
    float sx = 0.0f, sy = 0.0f;
    const float b[4] = {ld(V.b0 + k), ld(V.b1 + k), ld(V.b2 + k), ld(V.b3 + k)};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        uint32_t n = nbr(k, x, y, lw, lh, d);
        sx = sx + b[d] * ld(V.px + n);
        sy = sy + b[d] * ld(V.py + n);
    }
    const float dg = diagAt(V, k);
    const float pinx = pin ? pin[k] : 0.0f;
    return V2{ld(V.rx + k) - (sx - (dg + pinx) * ld(V.px + k)) * inv_h2,
              ld(V.ry + k) - (sy - (dg + 0.0f) * ld(V.py + k)) * inv_h2};
}

// restrictLevel's values of level-l cell (cx, cy) from level l - 1, stored
// as TU (fluid.wgsl:2342-2377): the density and, with `res`, the restricted
// residuals; all 0 in a block not worked on.  The four finer cells' words
// are all loaded before any is used (a cell past the level's edge reads
// the level's first cell and is then left out; a cell not liquid has its
// residual worked and dropped), so their loads are in flight together; the
// sums then take the liquid cells in the reference's order.
template <class VT>
__device__ __forceinline__ void restrictedFrom(const Dev& D, const FastW& F, const W& w, uint32_t l, const VT& U, int cx,
                                               int cy, bool res, float& rho_o, float& rx_o, float& ry_o) {
    const int span = 1 << l;
    if (span <= BLOCK) {
        I2 b{cx * span / BLOCK, cy * span / BLOCK};
        if (w.inBlocks(b) && (D.blocks[w.stateSlot(w.blockIndex(b))] & ACTIVE) == 0u) {
            rho_o = 0.0f;
            rx_o = 0.0f;
            ry_o = 0.0f;
            return;
        }
    }
    const int uw = (int)D.level_w[l - 1], uh = (int)D.level_h[l - 1];
    const float inv_h2 = 1.0f / (float)(1u << (2u * (l - 1u)));
    const float* pin = l == 1u ? F.pin : nullptr;
    float rq[4];
    V2 eq[4];
    bool inq[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int kx = 2 * cx + (q & 1), ky = 2 * cy + (q >> 1);
        inq[q] = kx < uw && ky < uh;  // rhoAt outside the level: -1
        const int sx = inq[q] ? kx : 0, sy = inq[q] ? ky : 0;
        const uint32_t k = (uint32_t)sy * (uint32_t)uw + (uint32_t)sx;
        rq[q] = ld(U.rho + k);
        eq[q] = res ? residualStored(U, pin, k, sx, sy, uw, uh, inv_h2) : V2{0.0f, 0.0f};
    }
    float fluid = 0.0f, sum = 0.0f, rx = 0.0f, ry = 0.0f;
    bool air = false;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (!inq[q]) continue;
        const float rho = rq[q];
        if (rho == 0.0f) air = true;
        else if (rho > 0.0f) {
            fluid = fluid + 1.0f;
            sum = sum + rho;
            if (res) {
                rx = rx + eq[q].x;
                ry = ry + eq[q].y;
            }
        }
    }
    const float rho = air ? 0.0f : (fluid > 0.0f ? sum / fluid : -1.0f);
    rho_o = rho;
    rx_o = rho > 0.0f ? rx * 0.25f : 0.0f;
    ry_o = rho > 0.0f ? ry * 0.25f : 0.0f;
}

// restrictedFrom for level l of a form whose levels store operator T: from
// level 0 as its smoother reads it, or from level l - 1.
template <class T>
__device__ __forceinline__ void restrictedAt(const Dev& D, const FastW& F, const W& w, uint32_t l, int cx, int cy,
                                             bool res, float& rho_o, float& rx_o, float& ry_o) {
    if (l == 1u) restrictedFrom(D, F, w, l, lref0<T>(F), cx, cy, res, rho_o, rx_o, ry_o);
    else restrictedFrom(D, F, w, l, lref<T>(F, l - 1u), cx, cy, res, rho_o, rx_o, ry_o);
}

// One coarse cell of restrictLevel, level l (stored as TV) from l - 1
// (stored as TU): the cell's values, its potentials zeroed.
template <class T>
__device__ void restrictCellT(const Dev& D, const FastW& F, const W& w, uint32_t l, uint32_t j) {
    const int lw = (int)D.level_w[l];
    const LRef<T> V = lref<T>(F, l);
    float rho, rx, ry;
    restrictedAt<T>(D, F, w, l, (int)(j % (uint32_t)lw), (int)(j / (uint32_t)lw), true, rho, rx, ry);
    st(V.px + j, 0.0f);
    st(V.py + j, 0.0f);
    st(V.rx + j, rx);
    st(V.ry + j, ry);
    st(V.rho + j, rho);
}
// Level l from l - 1 with the levels stored as T (level 0 always f32).
template <class T = float>
__device__ __forceinline__ void restrictCell(const Dev& D, const FastW& F, const W& w, uint32_t l, uint32_t j) {
    restrictCellT<T>(D, F, w, l, j);
}

// One cell of smoothAt (fluid.wgsl:2318-2334) on level l >= 1, the
// coefficients worked out on the step's first iteration and kept.
template <class T = float>
__device__ void smoothCell(const Dev& D, const FastW& F, uint32_t l, int color, bool first, uint32_t j) {
    const int lw = (int)D.level_w[l], lh = (int)D.level_h[l];
    const int cx = (int)(j % (uint32_t)lw), cy = (int)(j / (uint32_t)lw);
    if (((cx + cy) & 1) != color) return;
    const LRef<T> V = lref<T>(F, l);
    const float rho = ld(V.rho + j);
    if (rho <= 0.0f) return;
    float b[4];
    float dg;
    if (first) {
        dg = 0.0f;
        for (int d = 0; d < 4; d++) {
            b[d] = 0.0f;
            if (!nbrIn(cx, cy, lw, lh, d)) continue;
            float r = ld(V.rho + nbr(j, cx, cy, lw, lh, d));
            if (r < 0.0f) continue;
            b[d] = faceBeta(rho, r);
            dg = dg + b[d];
        }
        st(V.b0 + j, b[0]); st(V.b1 + j, b[1]); st(V.b2 + j, b[2]); st(V.b3 + j, b[3]);
        if (V.diag) st(V.diag + j, dg);
        // worked in what is stored, as later iterations read it
        b[0] = ld(V.b0 + j); b[1] = ld(V.b1 + j); b[2] = ld(V.b2 + j); b[3] = ld(V.b3 + j);
        dg = diagAt(V, j);
    } else {
        b[0] = ld(V.b0 + j); b[1] = ld(V.b1 + j); b[2] = ld(V.b2 + j); b[3] = ld(V.b3 + j);
        dg = diagAt(V, j);
    }
    if (dg <= 0.0f) return;
    float sx = 0.0f, sy = 0.0f;
#pragma unroll
    for (int d = 0; d < 4; d++) {
        uint32_t n = nbr(j, cx, cy, lw, lh, d);
        sx = sx + b[d] * ld(V.px + n);
        sy = sy + b[d] * ld(V.py + n);
    }
    const float h2 = (float)(1u << (2u * l));
    const float ex = ld(V.px + j), ey = ld(V.py + j);
    st(V.px + j, mixf(ex, (sx - h2 * ld(V.rx + j)) / dg, 1.0f));
    st(V.py + j, mixf(ey, (sy - h2 * ld(V.ry + j)) / dg, 1.0f));
}

// prolonged (fluid.wgsl:2478-2497) from level l + 1's arrays.  The four
// coarse cells' words are loaded before any is used (a cell past the
// level's edge reads a clamped one and is left out), then weighed in the
// reference's order.
template <class T, class P>
__device__ __forceinline__ V2 prolongedFrom(const T* rho, const P* px, const P* py, int lw, int lh, int cx, int cy) {
    const int kx = cx / 2, ky = cy / 2;
    const int sx = (cx & 1) == 1 ? 1 : -1, sy = (cy & 1) == 1 ? 1 : -1;
    const int ox[4] = {0, sx, 0, sx}, oy[4] = {0, 0, sy, sy};
    const float wt[4] = {9.0f, 3.0f, 3.0f, 1.0f};
    float rq[4], xq[4], yq[4];
    bool inq[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int ax_ = kx + ox[q], ay_ = ky + oy[q];
        inq[q] = !(ax_ < 0 || ay_ < 0 || ax_ >= lw || ay_ >= lh);
        const uint32_t k = inq[q] ? (uint32_t)ay_ * (uint32_t)lw + (uint32_t)ax_ : 0u;
        rq[q] = ld(rho + k);
        xq[q] = ld(px + k);
        yq[q] = ld(py + k);
    }
    float ax = 0.0f, ay = 0.0f, weight = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (!inq[q]) continue;
        const float r = rq[q];
        if (r < 0.0f) continue;
        weight = weight + wt[q];
        if (r > 0.0f) {
            ax = ax + wt[q] * xq[q];
            ay = ay + wt[q] * yq[q];
        }
    }
    const float ww = fmaxf(weight, 1e-6f);
    return V2{ax / ww, ay / ww};
}

// One cell of prolong (fluid.wgsl:2459-2470), level l from l + 1.
template <class T = float>
__device__ void prolongCell(const Dev& D, const FastW& F, uint32_t l, uint32_t j) {
    const int lw = (int)D.level_w[l];
    const LRef<T> V = lref<T>(F, l);
    if (ld(V.rho + j) <= 0.0f) return;
    const LRef<T> U = lref<T>(F, l + 1u);
    V2 e = prolongedFrom(U.rho, U.px, U.py, (int)D.level_w[l + 1], (int)D.level_h[l + 1], (int)(j % (uint32_t)lw),
                         (int)(j / (uint32_t)lw));
    st(V.px + j, ld(V.px + j) + e.x);
    st(V.py + j, ld(V.py + j) + e.y);
}

// ---------------------------------------------------------------- level tiles
//
// The levels above the coarse kernel's, a 16x16 tile of level l a 256-thread
// CTA, each pass of one level in one kernel: on the way down the tile's
// restriction and both colours of smoothing, on the way up its
// prolongation and both colours.  A tile works a ring of 2 cells around
// itself again (its neighbours' work, the same arithmetic on the same
// inputs, so the same bits): the red sweep on the ring of 1 reads the ring
// of 2, the black sweep on the tile reads the ring of 1.  Shared-memory
// arrays are 20 x 20, tile cell (0, 0) at (2, 2).

constexpr int LT = 16, LR = LT + 4, LRR = LR * LR;

__device__ __forceinline__ int lsi(int ix, int iy) { return (iy + 2) * LR + (ix + 2); }

// The shared index of neighbour d of tile cell (ix, iy) at level cell
// (cx, cy): clamped onto the cell past the level's edge, as nbr.
__device__ __forceinline__ int lsn(int ix, int iy, int cx, int cy, int lw, int lh, int d) {
    if (!nbrIn(cx, cy, lw, lh, d)) return lsi(ix, iy);
    switch (d) {
    case 0: return lsi(ix - 1, iy);
    case 1: return lsi(ix + 1, iy);
    case 2: return lsi(ix, iy - 1);
    default: return lsi(ix, iy + 1);
    }
}

// A value as a level of T stores it and reads it back.
__device__ __forceinline__ float asStored(float v, float) { return v; }
__device__ __forceinline__ float asStored(float v, __half) { return __half2float(__float2half_rn(v)); }

struct LevelTile {
    float rho[LRR], px[LRR], py[LRR], rx[LRR], ry[LRR], b[4][LRR], dg[LRR];
};

// One colour's sweep of smoothAt (fluid.wgsl:2318-2334) over tile cell
// (ix, iy) held in the tile's arrays.
__device__ __forceinline__ void tileSweepCell(LevelTile& t, int ix, int iy, int cx, int cy, int lw, int lh, float h2) {
    const int i = lsi(ix, iy);
    if (t.rho[i] <= 0.0f) return;
    const float dg = t.dg[i];
    if (dg <= 0.0f) return;
    float sx = 0.0f, sy = 0.0f;
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const int n = lsn(ix, iy, cx, cy, lw, lh, d);
        sx = sx + t.b[d][i] * t.px[n];
        sy = sy + t.b[d][i] * t.py[n];
    }
    t.px[i] = mixf(t.px[i], (sx - h2 * t.rx[i]) / dg, SMOOTH_OMEGA);
    t.py[i] = mixf(t.py[i], (sy - h2 * t.ry[i]) / dg, SMOOTH_OMEGA);
}

// The red sweep over the tile's ring of 1, the black over the tile itself.
__device__ __forceinline__ void tileSmooth(LevelTile& t, int x0, int y0, int lw, int lh, float h2) {
    for (int k = (int)threadIdx.x; k < (LT + 2) * (LT + 2); k += (int)blockDim.x) {
        const int ix = k % (LT + 2) - 1, iy = k / (LT + 2) - 1, cx = x0 + ix, cy = y0 + iy;
        if (cx < 0 || cy < 0 || cx >= lw || cy >= lh || ((cx + cy) & 1) != 0) continue;
        tileSweepCell(t, ix, iy, cx, cy, lw, lh, h2);
    }
    __syncthreads();
    if (threadIdx.x >= (unsigned)(LT * LT)) return;  // a wide CTA's threads past the tile's cells
    const int ix = (int)threadIdx.x % LT, iy = (int)threadIdx.x / LT, cx = x0 + ix, cy = y0 + iy;
    if (cx < lw && cy < lh && ((cx + cy) & 1) == 1) tileSweepCell(t, ix, iy, cx, cy, lw, lh, h2);
}

// Down, level l: restrictLevel, then smoothRed and smoothBlack when the
// world smooths level l (l < its coarse kernel's first level; else the
// restriction alone).  The coefficients of each liquid cell of the ring of 1
// from the densities (as the step's first iteration works and stores them,
// and later ones read them back), stored by the tile's own cells on the
// first iteration.
template <bool ONE, class T, int NT = 256>
__global__ void __launch_bounds__(NT, NT == 256 ? 4 : 2) k_fDown(Batch Bt, const __grid_constant__ WorldSrc<ONE> src, uint32_t l) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    __shared__ LevelTile t;
    FOR_ITEMS(Bt, L_RES + l - 1u, it) {
        FAST_ITEM(Bt, it, D, F, w, tile);
        if (D.st->cont == 0u) continue;
        const int lw = (int)D.level_w[l], lh = (int)D.level_h[l], tw = (lw + LT - 1) / LT;
        const int x0 = (int)(tile % (uint32_t)tw) * LT, y0 = (int)(tile / (uint32_t)tw) * LT;
        if (l >= F.lc) {
            const int cx = x0 + (int)threadIdx.x % LT, cy = y0 + (int)threadIdx.x / LT;
            if (threadIdx.x < (unsigned)(LT * LT) && cx < lw && cy < lh)
                restrictCell<T>(D, F, w, l, (uint32_t)(cy * lw + cx));
            continue;
        }
        const LRef<T> V = lref<T>(F, l);
        const bool first = D.st->cycle == 0u;
        for (int k = (int)threadIdx.x; k < LRR; k += (int)blockDim.x) {
            const int ix = k % LR - 2, iy = k / LR - 2, cx = x0 + ix, cy = y0 + iy;
            float rho = -1.0f, rx = 0.0f, ry = 0.0f;
            if (cx >= 0 && cy >= 0 && cx < lw && cy < lh) {
                const bool res = ix >= -1 && iy >= -1 && ix <= LT && iy <= LT;
                restrictedAt<T>(D, F, w, l, cx, cy, res, rho, rx, ry);
            }
            t.rho[k] = asStored(rho, T());
            t.rx[k] = rx;
            t.ry[k] = ry;
            t.px[k] = 0.0f;
            t.py[k] = 0.0f;
        }
        __syncthreads();
        for (int k = (int)threadIdx.x; k < (LT + 2) * (LT + 2); k += (int)blockDim.x) {
            const int ix = k % (LT + 2) - 1, iy = k / (LT + 2) - 1, cx = x0 + ix, cy = y0 + iy;
            if (cx < 0 || cy < 0 || cx >= lw || cy >= lh) continue;
            const int i = lsi(ix, iy);
            const float rho = t.rho[i];
            if (rho <= 0.0f) continue;
            float b[4];
            float dg = 0.0f;
#pragma unroll
            for (int d = 0; d < 4; d++) {
                b[d] = 0.0f;
                if (!nbrIn(cx, cy, lw, lh, d)) continue;
                const float r = t.rho[lsn(ix, iy, cx, cy, lw, lh, d)];
                if (r < 0.0f) continue;
                b[d] = faceBeta(rho, r);
                dg = dg + b[d];
            }
            const bool own = ix >= 0 && iy >= 0 && ix < LT && iy < LT;
            if (first && own) {
                const uint32_t j = (uint32_t)(cy * lw + cx);
                st(V.b0 + j, b[0]); st(V.b1 + j, b[1]); st(V.b2 + j, b[2]); st(V.b3 + j, b[3]);
                if (V.diag) st(V.diag + j, dg);
            }
#pragma unroll
            for (int d = 0; d < 4; d++) t.b[d][i] = asStored(b[d], T());
            // the diagonal as diagAt reads it: stored in f32, the rounded
            // coefficients' sum in binary16
            t.dg[i] = V.diag ? dg : ((t.b[0][i] + t.b[1][i]) + t.b[2][i]) + t.b[3][i];
        }
        __syncthreads();
        tileSmooth(t, x0, y0, lw, lh, (float)(1u << (2u * l)));
        if (threadIdx.x < (unsigned)(LT * LT)) {
            const int ix = (int)threadIdx.x % LT, iy = (int)threadIdx.x / LT, cx = x0 + ix, cy = y0 + iy;
            if (cx < lw && cy < lh) {
                const uint32_t j = (uint32_t)(cy * lw + cx);
                const int i = lsi(ix, iy);
                st(V.px + j, t.px[i]);
                st(V.py + j, t.py[i]);
                st(V.rx + j, t.rx[i]);
                st(V.ry + j, t.ry[i]);
                st(V.rho + j, t.rho[i]);
            }
        }
        __syncthreads();  // the tile's arrays are free for the next item
    }
}

// Up, level l (< the coarse kernel's first): prolong from level l + 1
// (fluid.wgsl:2459-2497), then smoothRed and smoothBlack with the stored
// coefficients.  The way down's potentials are read from px, py (the ring
// too) and the results go to ux, uy, so no CTA reads a cell that another
// writes in the same launch; level l + 1's results are its ux, uy.
template <bool ONE, class T, int NT = 256>
__global__ void __launch_bounds__(NT, NT == 256 ? 4 : 2) k_fUp(Batch Bt, const __grid_constant__ WorldSrc<ONE> src, uint32_t l) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    __shared__ LevelTile t;
    FOR_ITEMS(Bt, L_SM + l - 1u, it) {
        FAST_ITEM(Bt, it, D, F, w, tile);
        if (D.st->cont == 0u) continue;
        const int lw = (int)D.level_w[l], lh = (int)D.level_h[l], tw = (lw + LT - 1) / LT;
        const int x0 = (int)(tile % (uint32_t)tw) * LT, y0 = (int)(tile / (uint32_t)tw) * LT;
        const LRef<T> V = lref<T>(F, l);
        const T* urho = lref<T>(F, l + 1u).rho;
        const auto* lux = upx<T>(F, l + 1u);
        const auto* luy = upy<T>(F, l + 1u);
        const int uw = (int)D.level_w[l + 1], uh = (int)D.level_h[l + 1];
        for (int k = (int)threadIdx.x; k < LRR; k += (int)blockDim.x) {
            const int ix = k % LR - 2, iy = k / LR - 2, cx = x0 + ix, cy = y0 + iy;
            float rho = -1.0f, px = 0.0f, py = 0.0f;
            if (cx >= 0 && cy >= 0 && cx < lw && cy < lh) {
                // every word the cell may need loaded before any is used (a
                // cell not liquid drops them)
                const uint32_t j = (uint32_t)(cy * lw + cx);
                const bool ring1 = ix >= -1 && iy >= -1 && ix <= LT && iy <= LT;
                rho = ld(V.rho + j);
                px = ld(V.px + j);
                py = ld(V.py + j);
                const V2 e = prolongedFrom(urho, lux, luy, uw, uh, cx, cy);
                float rx = 0.0f, ry = 0.0f, b0 = 0.0f, b1 = 0.0f, b2 = 0.0f, b3 = 0.0f, dg = 0.0f;
                if (ring1) {
                    rx = ld(V.rx + j);
                    ry = ld(V.ry + j);
                    b0 = ld(V.b0 + j);
                    b1 = ld(V.b1 + j);
                    b2 = ld(V.b2 + j);
                    b3 = ld(V.b3 + j);
                    dg = diagAt(V, j);
                }
                if (rho > 0.0f) {
                    px = px + e.x;
                    py = py + e.y;
                    if (ring1) {
                        t.rx[k] = rx;
                        t.ry[k] = ry;
                        t.b[0][k] = b0;
                        t.b[1][k] = b1;
                        t.b[2][k] = b2;
                        t.b[3][k] = b3;
                        t.dg[k] = dg;
                    }
                }
            }
            t.rho[k] = rho;
            t.px[k] = px;
            t.py[k] = py;
        }
        __syncthreads();
        tileSmooth(t, x0, y0, lw, lh, (float)(1u << (2u * l)));
        if (threadIdx.x < (unsigned)(LT * LT)) {
            const int ix = (int)threadIdx.x % LT, iy = (int)threadIdx.x / LT, cx = x0 + ix, cy = y0 + iy;
            const int i = lsi(ix, iy);
            if (cx < lw && cy < lh && t.rho[i] > 0.0f) {
                const uint32_t j = (uint32_t)(cy * lw + cx);
                st(upx<T>(F, l) + j, t.px[i]);
                st(upy<T>(F, l) + j, t.py[i]);
            }
        }
        __syncthreads();
    }
}

// Named barrier over the first `count` threads (a multiple of 32).
__device__ __forceinline__ void barSub(uint32_t count) { asm volatile("bar.sync 1, %0;" ::"r"(count) : "memory"); }

// Level l (lc <= l <= levels) of the one-CTA kernel's shared memory: nine
// arrays of the level's cells from sm + off[l]: the potentials, the
// right-hand sides, the densities and the four face coefficients.
constexpr uint32_t SLV_ARRAYS = 9;
struct SLv {
    float *px, *py, *rx, *ry, *rho, *b0, *b1, *b2, *b3;
    int w, h;
    uint32_t mw;  // ceil(2^32 / w) (0 for w = 1): j / w = umulhi(j, mw) for the level's indices
};
__device__ __forceinline__ SLv slv(float* sm, const uint32_t* off, const Dev& D, uint32_t l) {
    const int n = (int)(D.level_w[l] * D.level_h[l]);
    float* p = sm + off[l];
    const uint32_t w = D.level_w[l];
    return SLv{p,         p + n,     p + 2 * n, p + 3 * n, p + 4 * n, p + 5 * n,
               p + 6 * n, p + 7 * n, p + 8 * n, (int)w, (int)D.level_h[l], w == 1u ? 0u : 0xffffffffu / w + 1u};
}
// The row of index j < 2 n of level V: j / w by a multiply-high with
// ceil(2^32 / w), exact while j w < 2^32 (the coarse kernel's levels hold at
// most 4096 cells), in place of an integer division's instruction sequence.
__device__ __forceinline__ int slvRow(const SLv& V, int j) {
    return V.w == 1 ? j : (int)__umulhi((uint32_t)j, V.mw);
}

// The face coefficients of level V's cells (smoothAt's stencil,
// fluid.wgsl:2318-2334): faceBeta to each neighbour inside the level whose
// density is not negative, else 0; all 0 for a cell that is not liquid.
__device__ void slv_coefficients(const SLv& V, int tid, int nt) {
    const int n = V.w * V.h;
    for (int j = tid; j < n; j += nt) {
        const int cy = slvRow(V, j), cx = j - cy * V.w;
        const float rho = V.rho[j];
        float b[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (rho > 0.0f) {
#pragma unroll
            for (int d = 0; d < 4; d++) {
                if (!nbrIn(cx, cy, V.w, V.h, d)) continue;
                const float r = V.rho[nbr((uint32_t)j, cx, cy, V.w, V.h, d)];
                if (r >= 0.0f) b[d] = faceBeta(rho, r);
            }
        }
        V.b0[j] = b[0];
        V.b1[j] = b[1];
        V.b2[j] = b[2];
        V.b3[j] = b[3];
    }
}

// The stencil's sums at liquid cell j from the stored coefficients: the
// sums of the neighbours taken in order, each beta times the neighbour's
// potential, and the betas' sum.  A neighbour the stencil skips has beta 0
// and its index clamped onto j, so adding its term changes no bit.
__device__ __forceinline__ void slv_stencil(const SLv& V, int j, int cx, int cy, float* sx, float* sy, float* dg) {
    const float b0 = V.b0[j], b1 = V.b1[j], b2 = V.b2[j], b3 = V.b3[j];
    const uint32_t n0 = nbr((uint32_t)j, cx, cy, V.w, V.h, 0), n1 = nbr((uint32_t)j, cx, cy, V.w, V.h, 1);
    const uint32_t n2 = nbr((uint32_t)j, cx, cy, V.w, V.h, 2), n3 = nbr((uint32_t)j, cx, cy, V.w, V.h, 3);
    *sx = (((0.0f + b0 * V.px[n0]) + b1 * V.px[n1]) + b2 * V.px[n2]) + b3 * V.px[n3];
    *sy = (((0.0f + b0 * V.py[n0]) + b1 * V.py[n1]) + b2 * V.py[n2]) + b3 * V.py[n3];
    *dg = (((0.0f + b0) + b1) + b2) + b3;
}

// One sweep of one colour over level V (smoothRed/Black, fluid.wgsl:2318-
// 2334, or the solve's SOR sweeps with omega): a thread per cell of that
// colour.  Of the cells 2k and 2k + 1 exactly one has each colour (in a row,
// or across a row's end when the width is odd), so pair k gives the cell.
__device__ void slv_sweep(const SLv& V, uint32_t l, int color, float omega, int tid, int nt) {
    const int n = V.w * V.h, pairs = (n + 1) / 2;
    const float h2 = (float)(1u << (2u * l));
    for (int k = tid; k < pairs; k += nt) {
        int j = 2 * k, cy = slvRow(V, j), cx = j - cy * V.w;
        if (((cx + cy) & 1) != color) {
            j++;
            if (++cx == V.w) {
                cx = 0;
                cy++;
            }
        }
        if (j >= n) continue;
        if (V.rho[j] <= 0.0f) continue;
        float sx, sy, dg;
        slv_stencil(V, j, cx, cy, &sx, &sy, &dg);
        if (dg <= 0.0f) continue;
        V.px[j] = mixf(V.px[j], (sx - h2 * V.rx[j]) / dg, omega);
        V.py[j] = mixf(V.py[j], (sy - h2 * V.ry[j]) / dg, omega);
    }
}

__device__ void slv_smooth(const SLv& V, uint32_t l, int tid, int nt) {
    for (int color = 0; color < 2; color++) {
        slv_sweep(V, l, color, SMOOTH_OMEGA, tid, nt);
        __syncthreads();
    }
}

// A coarsest-level cell of the solve, held in registers: its index, its
// four neighbours (clamped, nbr), their coefficients, the diagonal's FP64
// reciprocal (quotBy: the 80 sweeps' divisions by it), h^2 times its
// right-hand sides, and whether it is updated (a liquid cell with a
// positive diagonal, j < n).
struct SolveCell {
    uint32_t j, nb[4];
    float b[4], dg, hx, hy;
    double rd;
    int color;
    bool mine;
};
__device__ __forceinline__ SolveCell solveCell(const SLv& V, int j, int n, float h2) {
    SolveCell c;
    const int cy = slvRow(V, j), cx = j - cy * V.w;
    c.j = (uint32_t)j;
    c.color = (cx + cy) & 1;
    float r0 = -1.0f;
    c.dg = 0.0f;
    c.hx = 0.0f;
    c.hy = 0.0f;
#pragma unroll
    for (int d = 0; d < 4; d++) {
        c.b[d] = 0.0f;
        c.nb[d] = 0u;
    }
    if (j < n) {
        r0 = V.rho[j];
        c.hx = h2 * V.rx[j];
        c.hy = h2 * V.ry[j];
        c.b[0] = V.b0[j]; c.b[1] = V.b1[j]; c.b[2] = V.b2[j]; c.b[3] = V.b3[j];
#pragma unroll
        for (int d = 0; d < 4; d++) c.nb[d] = nbr((uint32_t)j, cx, cy, V.w, V.h, d);
        c.dg = (((0.0f + c.b[0]) + c.b[1]) + c.b[2]) + c.b[3];
    }
    c.mine = j < n && r0 > 0.0f && c.dg > 0.0f;
    c.rd = recipOf(c.dg);
    return c;
}
// One SOR update (omega 1.8) of a solve cell from its neighbours' potentials.
__device__ __forceinline__ void solveUpdate(const SLv& V, const SolveCell& c) {
    if (!c.mine) return;
    float* px = V.px;
    float* py = V.py;
    float sx = c.b[0] * px[c.nb[0]] + c.b[1] * px[c.nb[1]] + c.b[2] * px[c.nb[2]] + c.b[3] * px[c.nb[3]];
    float sy = c.b[0] * py[c.nb[0]] + c.b[1] * py[c.nb[1]] + c.b[2] * py[c.nb[2]] + c.b[3] * py[c.nb[3]];
    px[c.j] = mixf(px[c.j], quotBy(sx - c.hx, c.rd), OMEGA);
    py[c.j] = mixf(py[c.j], quotBy(sy - c.hy, c.rd), OMEGA);
}

// The levels from lc (in sm from offsets off[]: just loaded, or restricted
// already) down to the coarsest and back up to lc: each level's
// coefficients worked out once its densities are in place, smoothRed/Black,
// restrictLevel, solve (40 SOR sweep pairs, omega 1.8), prolong
// (fluid.wgsl:2318-2470); the result in level lc's px, py.  Every thread of
// the CTA takes part.
__device__ void coarseCore(const Dev& D, const W& w, uint32_t lc, float* sm, const uint32_t* off) {
    const uint32_t L = D.levels;
    const int tid = (int)threadIdx.x, nt = (int)blockDim.x;
    for (uint32_t l = lc; l <= L; l++) {
        const SLv V = slv(sm, off, D, l);
        const int n = V.w * V.h;
        if (l > lc) {
            const SLv U = slv(sm, off, D, l - 1u);
            const int span = 1 << l;
            // 1 / h^2 of level l - 1: a power of two, so the product is the
            // quotient's bits
            const float inv_h2u = 1.0f / (float)(1u << (2u * (l - 1u)));
            for (int j = tid; j < n; j += nt) {
                const int cy = slvRow(V, j), cx = j - cy * V.w;
                if (span <= BLOCK) {
                    I2 b{cx * span / BLOCK, cy * span / BLOCK};
                    if (w.inBlocks(b) && (D.blocks[w.stateSlot(w.blockIndex(b))] & ACTIVE) == 0u) {
                        V.px[j] = 0.0f; V.py[j] = 0.0f; V.rx[j] = 0.0f; V.ry[j] = 0.0f; V.rho[j] = 0.0f;
                        continue;
                    }
                }
                float fluid = 0.0f, sum = 0.0f, rx = 0.0f, ry = 0.0f;
                bool air = false;
                for (int q = 0; q < 4; q++) {
                    int kx = 2 * cx + (q & 1), ky = 2 * cy + (q >> 1);
                    if (kx >= U.w || ky >= U.h) continue;
                    int k = ky * U.w + kx;
                    float rho = U.rho[k];
                    if (rho == 0.0f) air = true;
                    else if (rho > 0.0f) {
                        float sx, sy, dg;
                        slv_stencil(U, k, kx, ky, &sx, &sy, &dg);
                        fluid = fluid + 1.0f;
                        sum = sum + rho;
                        rx = rx + (U.rx[k] - (sx - (dg + 0.0f) * U.px[k]) * inv_h2u);
                        ry = ry + (U.ry[k] - (sy - (dg + 0.0f) * U.py[k]) * inv_h2u);
                    }
                }
                const float rho = air ? 0.0f : (fluid > 0.0f ? sum / fluid : -1.0f);
                V.px[j] = 0.0f;
                V.py[j] = 0.0f;
                V.rx[j] = rho > 0.0f ? rx * 0.25f : 0.0f;
                V.ry[j] = rho > 0.0f ? ry * 0.25f : 0.0f;
                V.rho[j] = rho;
            }
            __syncthreads();
        }
        slv_coefficients(V, tid, nt);
        __syncthreads();
        if (l < L) slv_smooth(V, l, tid, nt);
    }
    // solve: the coarsest level.  When its cells fit the CTA, thread k of the
    // first warps holds cells 2k and 2k + 1, one of each colour (in a row, or
    // across a row's end when the width is odd), their coefficients in
    // registers across the sweeps: every thread of those warps updates a
    // cell each sweep, and only they are synchronised (a named barrier over
    // npair <= blockDim threads); else a thread per cell of the swept
    // colour, the CTA synchronised.
    {
        const SLv V = slv(sm, off, D, L);
        const int n = min(V.w * V.h, (int)WIG_MG_COARSEST);
        const float h2 = (float)(1u << (2u * L));
        const int pairs = (n + 1) / 2;
        const uint32_t npair = (uint32_t)((pairs + 31) & ~31);
        if (npair <= (uint32_t)nt) {
            if (tid < (int)npair) {
                SolveCell c0 = solveCell(V, 2 * tid, n, h2), c1 = solveCell(V, 2 * tid + 1, n, h2);
                // c0 the colour-0 cell, c1 the colour-1 one
                if (c0.color != 0) {
                    const SolveCell t = c0;
                    c0 = c1;
                    c1 = t;
                }
                for (int s = 0; s < COARSE_SWEEPS; s++) {
                    solveUpdate(V, c0);
                    barSub(npair);
                    solveUpdate(V, c1);
                    barSub(npair);
                }
            }
        } else {
            for (int s = 0; s < 2 * COARSE_SWEEPS; s++) {
                slv_sweep(V, L, s & 1, OMEGA, tid, nt);
                __syncthreads();
            }
        }
        __syncthreads();
    }
    for (int l = (int)L - 1; l >= (int)lc; l--) {
        const SLv V = slv(sm, off, D, (uint32_t)l);
        const SLv U = slv(sm, off, D, (uint32_t)l + 1u);
        const int n = V.w * V.h;
        for (int j = tid; j < n; j += nt) {
            if (V.rho[j] <= 0.0f) continue;
            const int cy = slvRow(V, j);
            V2 e = prolongedFrom(U.rho, U.px, U.py, U.w, U.h, j - cy * V.w, cy);
            V.px[j] = V.px[j] + e.x;
            V.py[j] = V.py[j] + e.y;
        }
        __syncthreads();
        slv_smooth(V, (uint32_t)l, tid, nt);
    }
}

// The levels lc (restricted already, in the scratch) down to the coarsest and
// back up to lc, in one CTA's shared memory: smoothRed/Black, restrictLevel,
// solve (40 SOR sweep pairs, omega 1.8), prolong (fluid.wgsl:2318-2470).
// Each level's face coefficients are worked out once, when its densities
// are in place, and read by its sweeps and by the restriction below it.
// Level lc's results go to its ux, uy (`up`, the fast form) or back into its
// px, py (the persistent form).
template <class T = float>
__device__ void coarseLevels(const Dev& D, const FastW& F, const W& w, uint32_t lc, float* sm, uint32_t* off,
                             bool up) {
    const uint32_t L = D.levels;
    const int tid = (int)threadIdx.x, nt = (int)blockDim.x;
    if (tid == 0) {
        uint32_t o = 0;
        for (uint32_t l = lc; l <= L; l++) {
            off[l] = o;
            o += SLV_ARRAYS * D.level_w[l] * D.level_h[l];
        }
    }
    __syncthreads();
    {
        const SLv V = slv(sm, off, D, lc);
        const LRef<T> G = lref<T>(F, lc);
        const int n = V.w * V.h;
        for (int j = tid; j < n; j += nt) {
            V.px[j] = ld(G.px + j);
            V.py[j] = ld(G.py + j);
            V.rx[j] = ld(G.rx + j);
            V.ry[j] = ld(G.ry + j);
            V.rho[j] = ld(G.rho + j);
        }
        __syncthreads();
    }
    coarseCore(D, w, lc, sm, off);
    {
        const SLv V = slv(sm, off, D, lc);
        auto* ox = up ? upx<T>(F, lc) : lref<T>(F, lc).px;
        auto* oy = up ? upy<T>(F, lc) : lref<T>(F, lc).py;
        const int n = V.w * V.h;
        for (int j = tid; j < n; j += nt) {
            st(ox + j, V.px[j]);
            st(oy + j, V.py[j]);
        }
    }
}

template <bool ONE, class T>
__global__ void __launch_bounds__(1024) k_fCoarse(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    extern __shared__ float sm[];
    __shared__ uint32_t off[WIG_MG_LEVELS + 1];
    FOR_ITEMS(Bt, L_ONE, it) {
        FAST_ITEM(Bt, it, D, F, w, unused_);
        (void)unused_;
        if (D.st->cont == 0u) continue;
        coarseLevels<T>(D, F, w, F.lc, sm, off, true);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- the coarse levels on a cluster
//
// A single world whose coarse kernel starts at a level of more than
// COARSE_CTA_CELLS cells (at 1024 x 1024: 128 x 128, with the coarse_cells
// knob at 16384) runs its coarse levels on one thread-block cluster of
// CLUSTER_CTAS CTAs instead of one CTA, in their distributed shared memory.
// Each level of more than RANK0_CELLS cells is cut into strips of rows, a
// strip a CTA, its nine arrays (px, py, rx, ry, rho, b0..b3) in that CTA's
// shared memory at the same offsets in every CTA; a neighbour's row across a
// strip's edge is read from the owning CTA (cluster.map_shared_rank).  The
// levels of at most RANK0_CELLS cells are CTA 0's alone (coarseCore, as in
// the one-CTA kernel).  Every pass is the one-CTA kernel's, cell for cell, in
// the same arithmetic and order (the cells of a colour are independent), and
// a cluster barrier ends each pass whose results another CTA reads.  The
// levels it takes over from the tile kernels (the restrict-only launch of
// its first level stays) would each have been a launch of one wave of a few
// CTAs.
constexpr int CLUSTER_CTAS = 8;
constexpr uint32_t RANK0_CELLS = 1024;

enum { A_PX = 0, A_PY, A_RX, A_RY, A_RHO, A_B0, A_B1, A_B2, A_B3 };

// n / d for any 32-bit n, with mul = floor((2^32 - 1) / d): the multiply-high
// is the quotient or one below it.
__device__ __forceinline__ uint32_t divq(uint32_t n, uint32_t d, uint32_t mul) {
    uint32_t q = __umulhi(n, mul);
    if (n - q * d >= d) q += 1u;
    return q;
}

// A level cut into strips: this CTA's rows r0 .. r1 - 1 of rpr a CTA; array
// k of a CTA's rows at base + k n (n = rpr w floats).
struct DLv {
    float* base;
    int n, w, h, rpr, r0, r1;
    uint32_t wmul, rmul;
    __device__ float* a(int k) const { return base + k * n; }
};
// The strip levels' shared memory: level lc's from sm, each next level's
// after the one above it.
__host__ __device__ inline size_t stripFloats(uint32_t w, uint32_t h) {
    return (size_t)SLV_ARRAYS * ((h + CLUSTER_CTAS - 1) / CLUSTER_CTAS) * w;
}
__device__ __forceinline__ DLv dlv(float* sm, const Dev& D, uint32_t lc, uint32_t l, unsigned me) {
    for (uint32_t k = lc; k < l; k++) sm += stripFloats(D.level_w[k], D.level_h[k]);
    DLv V;
    V.base = sm;
    V.w = (int)D.level_w[l];
    V.h = (int)D.level_h[l];
    V.rpr = (V.h + CLUSTER_CTAS - 1) / CLUSTER_CTAS;
    V.n = V.rpr * V.w;
    V.r0 = min((int)me * V.rpr, V.h);
    V.r1 = min(V.r0 + V.rpr, V.h);
    V.wmul = 0xffffffffu / (uint32_t)V.w;
    V.rmul = 0xffffffffu / (uint32_t)V.rpr;
    return V;
}
// Row y of a strip level (its array 0; array k at + k n), in whichever CTA
// holds it.
__device__ __forceinline__ float* dlRow(const DLv& V, int y, unsigned me) {
    const unsigned o = divq((uint32_t)y, (uint32_t)V.rpr, V.rmul);
    float* p = V.base + (y - (int)o * V.rpr) * V.w;
    return o == me ? p : cooperative_groups::this_cluster().map_shared_rank(p, o);
}
// This CTA's own cell j (of (r1 - r0) w): its coordinates.
__device__ __forceinline__ void dlCell(const DLv& V, int j, int* x, int* y) {
    const int q = (int)divq((uint32_t)j, (uint32_t)V.w, V.wmul);
    *x = j - q * V.w;
    *y = V.r0 + q;
}

// slv_stencil of a strip level's cell (x, y) in row r (its rows above and
// below from whichever CTAs hold them): the neighbours clamped onto the cell
// past the level's edge (nbr), each beta times its potential, in order.
__device__ __forceinline__ void dl_stencil(const DLv& V, const float* r, int x, int y, unsigned me, float* sx, float* sy,
                                           float* dg) {
    const float* u = y > 0 ? dlRow(V, y - 1, me) : r;
    const float* d = y < V.h - 1 ? dlRow(V, y + 1, me) : r;
    const int xl = x > 0 ? x - 1 : x, xr = x < V.w - 1 ? x + 1 : x;
    const int n = V.n;
    const float b0 = r[A_B0 * n + x], b1 = r[A_B1 * n + x], b2 = r[A_B2 * n + x], b3 = r[A_B3 * n + x];
    *sx = (((0.0f + b0 * r[xl]) + b1 * r[xr]) + b2 * u[x]) + b3 * d[x];
    *sy = (((0.0f + b0 * r[n + xl]) + b1 * r[n + xr]) + b2 * u[n + x]) + b3 * d[n + x];
    *dg = (((0.0f + b0) + b1) + b2) + b3;
}

// slv_coefficients over this CTA's strip.
__device__ void dl_coefficients(const DLv& V, unsigned me) {
    const int n = (V.r1 - V.r0) * V.w;
    for (int j = (int)threadIdx.x; j < n; j += (int)blockDim.x) {
        int x, y;
        dlCell(V, j, &x, &y);
        const float* own = V.a(A_RHO);
        const float rho = own[j];
        float b[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (rho > 0.0f) {
            const float* u = y > 0 ? dlRow(V, y - 1, me) + A_RHO * V.n : nullptr;
            const float* d = y < V.h - 1 ? dlRow(V, y + 1, me) + A_RHO * V.n : nullptr;
            const float rn[4] = {x > 0 ? own[j - 1] : 0.0f, x < V.w - 1 ? own[j + 1] : 0.0f, u ? u[x] : 0.0f,
                                 d ? d[x] : 0.0f};
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (!nbrIn(x, y, V.w, V.h, q)) continue;
                if (rn[q] >= 0.0f) b[q] = faceBeta(rho, rn[q]);
            }
        }
        V.a(A_B0)[j] = b[0];
        V.a(A_B1)[j] = b[1];
        V.a(A_B2)[j] = b[2];
        V.a(A_B3)[j] = b[3];
    }
}

// slv_sweep of one colour over this CTA's strip: of its cells 2k and
// 2k + 1 exactly one has each colour, so pair k gives the cell.
__device__ void dl_sweep(const DLv& V, uint32_t l, int color, float omega, unsigned me) {
    const int n = (V.r1 - V.r0) * V.w, pairs = (n + 1) / 2;
    const float h2 = (float)(1u << (2u * l));
    for (int k = (int)threadIdx.x; k < pairs; k += (int)blockDim.x) {
        int j = 2 * k, x, y;
        dlCell(V, j, &x, &y);
        if (((x + y) & 1) != color) {
            j++;
            if (++x == V.w) {
                x = 0;
                y++;
            }
        }
        if (j >= n) continue;
        if (V.a(A_RHO)[j] <= 0.0f) continue;
        float* r = V.base + (j - x);
        float sx, sy, dg;
        dl_stencil(V, r, x, y, me, &sx, &sy, &dg);
        if (dg <= 0.0f) continue;
        float* px = V.a(A_PX);
        float* py = V.a(A_PY);
        px[j] = mixf(px[j], (sx - h2 * V.a(A_RX)[j]) / dg, omega);
        py[j] = mixf(py[j], (sy - h2 * V.a(A_RY)[j]) / dg, omega);
    }
}

// restrictLevel into coarse cell (cx, cy) of level l from strip level U
// (level l - 1), as coarseCore restricts: the stencil from U's stored
// coefficients.
__device__ __forceinline__ void dl_restricted(const Dev& D, const W& w, uint32_t l, const DLv& U, int cx, int cy, unsigned me,
                                              float* px, float* py, float* rx_o, float* ry_o, float* rho_o) {
    const int span = 1 << l;
    if (span <= BLOCK) {
        I2 b{cx * span / BLOCK, cy * span / BLOCK};
        if (w.inBlocks(b) && (D.blocks[w.stateSlot(w.blockIndex(b))] & ACTIVE) == 0u) {
            *px = 0.0f; *py = 0.0f; *rx_o = 0.0f; *ry_o = 0.0f; *rho_o = 0.0f;
            return;
        }
    }
    const float inv_h2u = 1.0f / (float)(1u << (2u * (l - 1u)));
    const int n = U.n;
    float fluid = 0.0f, sum = 0.0f, rx = 0.0f, ry = 0.0f;
    bool air = false;
    for (int q = 0; q < 4; q++) {
        const int kx = 2 * cx + (q & 1), ky = 2 * cy + (q >> 1);
        if (kx >= U.w || ky >= U.h) continue;
        const float* r = dlRow(U, ky, me);
        const float rho = r[A_RHO * n + kx];
        if (rho == 0.0f) air = true;
        else if (rho > 0.0f) {
            float sx, sy, dg;
            dl_stencil(U, r, kx, ky, me, &sx, &sy, &dg);
            fluid = fluid + 1.0f;
            sum = sum + rho;
            rx = rx + (r[A_RX * n + kx] - (sx - (dg + 0.0f) * r[kx]) * inv_h2u);
            ry = ry + (r[A_RY * n + kx] - (sy - (dg + 0.0f) * r[n + kx]) * inv_h2u);
        }
    }
    const float rho = air ? 0.0f : (fluid > 0.0f ? sum / fluid : -1.0f);
    *px = 0.0f;
    *py = 0.0f;
    *rx_o = rho > 0.0f ? rx * 0.25f : 0.0f;
    *ry_o = rho > 0.0f ? ry * 0.25f : 0.0f;
    *rho_o = rho;
}

// prolonged (fluid.wgsl:2478-2497) of fine cell (cx, cy) from strip level
// U: prolongedFrom's loads and weights, U's two rows from their CTAs.
__device__ __forceinline__ V2 dl_prolonged(const DLv& U, int cx, int cy, unsigned me) {
    const int kx = cx / 2, ky = cy / 2;
    const int sx = (cx & 1) == 1 ? 1 : -1, sy = (cy & 1) == 1 ? 1 : -1;
    const int ox[4] = {0, sx, 0, sx}, oy[4] = {0, 0, sy, sy};
    const float wt[4] = {9.0f, 3.0f, 3.0f, 1.0f};
    const bool row2 = ky + sy >= 0 && ky + sy < U.h;
    const float* r0 = dlRow(U, ky, me);
    const float* r1 = row2 ? dlRow(U, ky + sy, me) : r0;
    const int n = U.n;
    float rq[4], xq[4], yq[4];
    bool inq[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int ax_ = kx + ox[q], ay_ = ky + oy[q];
        inq[q] = !(ax_ < 0 || ay_ < 0 || ax_ >= U.w || ay_ >= U.h);
        const float* r = oy[q] == 0 ? r0 : r1;
        const int c = inq[q] ? ax_ : kx;
        rq[q] = r[A_RHO * n + c];
        xq[q] = r[c];
        yq[q] = r[n + c];
    }
    float ax = 0.0f, ay = 0.0f, weight = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (!inq[q]) continue;
        const float r = rq[q];
        if (r < 0.0f) continue;
        weight = weight + wt[q];
        if (r > 0.0f) {
            ax = ax + wt[q] * xq[q];
            ay = ay + wt[q] * yq[q];
        }
    }
    const float ww = fmaxf(weight, 1e-6f);
    return V2{ax / ww, ay / ww};
}

// The cluster's shared memory (floats a CTA) for a world from level lc: each
// strip level's rows of one CTA, then CTA 0's levels ls .. L; 0 when the
// coarsest level has more than RANK0_CELLS cells.
__host__ __device__ inline size_t clusterFloats(const uint32_t* lw, const uint32_t* lh, uint32_t lc, uint32_t L,
                                                uint32_t* ls_out) {
    size_t n = 0;
    uint32_t l = lc;
    for (; l <= L && lw[l] * lh[l] > RANK0_CELLS; l++) n += stripFloats(lw[l], lh[l]);
    if (ls_out) *ls_out = l;
    if (l > L) return 0;
    for (uint32_t k = l; k <= L; k++) n += (size_t)SLV_ARRAYS * lw[k] * lh[k];
    return n;
}

template <class T>
__global__ void __launch_bounds__(1024) k_fCoarseCluster(Batch Bt, const __grid_constant__ WorldSrc<true> src) {
    extern __shared__ float sm[];
    __shared__ uint32_t off[WIG_MG_LEVELS + 1];
    namespace cgs = cooperative_groups;
    cgs::cluster_group cl = cgs::this_cluster();
    const unsigned me = cl.block_rank();
    const World& Wd = src.w;
    const Dev& D = Wd.D;
    const FastW& F = Wd.S;
    const W w(D);
    (void)Bt;
    // every CTA reads the same word: all go on, or all return, together
    if (D.st->cont == 0u) return;
    const uint32_t lc = F.lc, L = D.levels;
    uint32_t ls = lc;
    clusterFloats(D.level_w, D.level_h, lc, L, &ls);
    // CTA 0's levels ls .. L after the strip levels lc .. ls - 1
    float* sm0 = sm;
    for (uint32_t l = lc; l < ls; l++) sm0 += stripFloats(D.level_w[l], D.level_h[l]);
    if (threadIdx.x == 0) {
        uint32_t o = 0;
        for (uint32_t l = ls; l <= L; l++) {
            off[l] = o;
            o += SLV_ARRAYS * D.level_w[l] * D.level_h[l];
        }
    }
    // level lc's rows from the scratch (restricted by the down kernel)
    {
        const DLv A = dlv(sm, D, lc, lc, me);
        const LRef<T> G = lref<T>(F, lc);
        const int n = (A.r1 - A.r0) * A.w;
        for (int j = (int)threadIdx.x; j < n; j += (int)blockDim.x) {
            const int g = A.r0 * A.w + j;
            A.a(A_PX)[j] = ld(G.px + g);
            A.a(A_PY)[j] = ld(G.py + g);
            A.a(A_RX)[j] = ld(G.rx + g);
            A.a(A_RY)[j] = ld(G.ry + g);
            A.a(A_RHO)[j] = ld(G.rho + g);
        }
    }
    cl.sync();
    // down the strip levels
    for (uint32_t l = lc; l < ls; l++) {
        const DLv A = dlv(sm, D, lc, l, me);
        if (l > lc) {
            const DLv U = dlv(sm, D, lc, l - 1u, me);
            const int n = (A.r1 - A.r0) * A.w;
            for (int j = (int)threadIdx.x; j < n; j += (int)blockDim.x) {
                int x, y;
                dlCell(A, j, &x, &y);
                dl_restricted(D, w, l, U, x, y, me, &A.a(A_PX)[j], &A.a(A_PY)[j], &A.a(A_RX)[j], &A.a(A_RY)[j],
                              &A.a(A_RHO)[j]);
            }
            cl.sync();
        }
        dl_coefficients(A, me);
        __syncthreads();
        dl_sweep(A, l, 0, SMOOTH_OMEGA, me);
        cl.sync();
        dl_sweep(A, l, 1, SMOOTH_OMEGA, me);
        cl.sync();
    }
    // CTA 0: level ls restricted from the last strip level, then the levels
    // below it and back up, in its own shared memory
    if (me == 0u) {
        const DLv U = dlv(sm, D, lc, ls - 1u, me);
        const SLv S = slv(sm0, off, D, ls);
        const int n = S.w * S.h;
        for (int j = (int)threadIdx.x; j < n; j += (int)blockDim.x) {
            const int cy = slvRow(S, j), cx = j - cy * S.w;
            dl_restricted(D, w, ls, U, cx, cy, me, &S.px[j], &S.py[j], &S.rx[j], &S.ry[j], &S.rho[j]);
        }
        __syncthreads();
        coarseCore(D, w, ls, sm0, off);
    }
    cl.sync();
    // up the strip levels: prolong from the level below (CTA 0's or a strip
    // level), then both colours
    for (int l = (int)ls - 1; l >= (int)lc; l--) {
        const DLv A = dlv(sm, D, lc, (uint32_t)l, me);
        const int n = (A.r1 - A.r0) * A.w;
        if (l + 1 == (int)ls) {
            // CTA 0's level ls, at offset 0 of its levels there
            const int lw = (int)D.level_w[ls], lh = (int)D.level_h[ls];
            const int nl = lw * lh;
            const float* b0 = cl.map_shared_rank(sm0, 0u);
            for (int j = (int)threadIdx.x; j < n; j += (int)blockDim.x) {
                if (A.a(A_RHO)[j] <= 0.0f) continue;
                int x, y;
                dlCell(A, j, &x, &y);
                const V2 e = prolongedFrom(b0 + 4 * nl, b0, b0 + nl, lw, lh, x, y);
                A.a(A_PX)[j] = A.a(A_PX)[j] + e.x;
                A.a(A_PY)[j] = A.a(A_PY)[j] + e.y;
            }
        } else {
            const DLv U = dlv(sm, D, lc, (uint32_t)l + 1u, me);
            for (int j = (int)threadIdx.x; j < n; j += (int)blockDim.x) {
                if (A.a(A_RHO)[j] <= 0.0f) continue;
                int x, y;
                dlCell(A, j, &x, &y);
                const V2 e = dl_prolonged(U, x, y, me);
                A.a(A_PX)[j] = A.a(A_PX)[j] + e.x;
                A.a(A_PY)[j] = A.a(A_PY)[j] + e.y;
            }
        }
        cl.sync();
        dl_sweep(A, (uint32_t)l, 0, SMOOTH_OMEGA, me);
        cl.sync();
        dl_sweep(A, (uint32_t)l, 1, SMOOTH_OMEGA, me);
        cl.sync();
    }
    // level lc's rows to its way-up potentials
    {
        const DLv A = dlv(sm, D, lc, lc, me);
        const int n = (A.r1 - A.r0) * A.w;
        auto* ox = upx<T>(F, lc);
        auto* oy = upy<T>(F, lc);
        for (int j = (int)threadIdx.x; j < n; j += (int)blockDim.x) {
            const int g = A.r0 * A.w + j;
            st(ox + g, A.a(A_PX)[j]);
            st(oy + g, A.a(A_PY)[j]);
        }
    }
}

// prolongFine (fluid.wgsl:2500-2512), and the rims for the relaxation after.
template <bool ONE, class T>
__global__ void k_fProlongFine(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        FAST_ITEM(Bt, it, D, F, w, wid);
        if (D.st->cont == 0u) continue;
        const Lvl& L0 = F.L[0];
        const T* urho = lref<T>(F, 1u).rho;
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        // the cell's words and the prolongation's loaded together, then used
        // for a liquid cell only
        const float rho = L0.rho[i], px0 = L0.px[i], py0 = L0.py[i];
        const V2 e = prolongedFrom(urho, upx<T>(F, 1u), upy<T>(F, 1u), (int)D.level_w[1], (int)D.level_h[1], c.x, c.y);
        if (rho > 0.0f) {
            float px = px0 + e.x, py = py0 + e.y;
            L0.px[i] = px;
            L0.py[i] = py;
            F.rimx[i] = px;
            F.rimy[i] = py;
        }
    }
}

// ================================================================ conjugate gradients

// cgRho + cgBeta (fluid.wgsl:2736-2764): four tiles a 256-thread CTA; the CTA
// that counts a world's last tile sums its blocks' partials (sumBlocks' order).
template <bool ONE>
__global__ void __launch_bounds__(256) k_fRhoBeta(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    __shared__ float sx[256], sy[256];
    __shared__ double s64[256], s64b[256];
    __shared__ float ux[2][128], uy[2][128];
    __shared__ double ex64[2][128], ey64[2][128];
    uint32_t pend_ = 0;  // tiles finished of the current world, not yet counted
    uint32_t par = 0;    // the tree buffers of this item
    FOR_ITEMS(Bt, L_ACT4, it) {
        FAST_ITEM(Bt, it, D, F, w, g);
        if (D.st->cont == 0u) continue;
        const bool f64 = D.st->f64 != 0u;
        const uint32_t cycle = D.st->cycle;
        const Lvl& L0 = F.L[0];
        const uint32_t na = w.activeCount();
        const uint32_t wid = g * 4u + (threadIdx.x >> 6);
        const bool valid = wid < na;
        float vx = 0.0f, vy = 0.0f;
        double ex = 0.0, ey = 0.0;
        if (valid) {
            I2 c = tileCell(w, wid);
            if (w.inWorld(c)) {
                uint32_t i = w.cellIndex(c);
                // loaded beside the density, not after it: one dependent
                // load fewer on the item's path
                const float rho = L0.rho[i], z = L0.px[i], r = F.R[i], q = F.Q[i];
                if (rho > 0.0f) {
                    vx = r * z;
                    vy = q * z;
                    ex = (double)r * (double)z;
                    ey = (double)q * (double)z;
                }
            }
        }
        // the f32 trees only without FP64 dots, which read none of them
        if (f64) {
            tilePut(ex64[par], ex);
            tilePut(ey64[par], ey);
        } else {
            tilePut(ux[par], vx);
            tilePut(uy[par], vy);
        }
        __syncthreads();
        float tx = 0.0f, ty = 0.0f;
        double dx = 0.0, dy = 0.0;
        if (f64) {
            dx = tileSum(ex64[par], ex);
            dy = tileSum(ey64[par], ey);
        } else {
            tx = tileSum(ux[par], vx);
            ty = tileSum(uy[par], vy);
        }
        par ^= 1u;
        if (valid && (threadIdx.x & 63u) == 0u) {
            const uint32_t b = w.blockIndex(w.activeBlock(wid));
            if (f64) {
                F.part64[2u * b] = dx;
                F.part64[2u * b + 1u] = dy;
            } else {
                F.part32[2u * b] = tx;
                F.part32[2u * b + 1u] = ty;
            }
        }
        pend_ += min(4u, na - g * 4u);
        if (flushTiles(Bt, g_it, e_it, it, pend_, &D.st->fdone[1], na)) {
            if (f64) {
                double rz, zq;
                sumBlocks256x2(w, F.part64, s64, s64b, &rz, &zq);
                if (threadIdx.x == 0) {
                    double beta = (cycle == 0u || D.st->pq <= 0.0) ? 0.0 : -zq / D.st->pq;
                    D.st->rz = rz;
                    D.st->beta = beta;
                }
            } else {
                float rz, zq;
                sumBlocks256x2(w, F.part32, sx, sy, &rz, &zq);
                if (threadIdx.x == 0) {
                    float beta = (cycle == 0u || D.st->pq32 <= 0.0f) ? 0.0f : -zq / D.st->pq32;
                    D.st->rz32 = rz;
                    D.st->beta32 = beta;
                }
            }
        }
    }
}

// cgDirection + cgApply + cgAlpha (fluid.wgsl:2767-2814): the direction p =
// z + beta p_old of the cell and of its liquid neighbours (worked again from
// their z and p_old, the same arithmetic), q = A p, and the tile trees of
// p q.  p_old is read from one of the two p arrays and p written to the
// other (by the iteration's parity), so no CTA reads a p that another
// writes in the launch.
template <bool ONE>
__global__ void __launch_bounds__(256) k_fApplyAlpha(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    __shared__ float sx[256];
    __shared__ double s64[256];
    __shared__ float ux[2][128];
    __shared__ double ex64[2][128];
    uint32_t pend_ = 0;  // tiles finished of the current world, not yet counted
    uint32_t par = 0;    // the tree buffers of this item
    FOR_ITEMS(Bt, L_ACT4, it) {
        FAST_ITEM(Bt, it, D, F, w, g);
        if (D.st->cont == 0u) continue;
        const bool f64 = D.st->f64 != 0u;
        const float beta = D.st->beta32;
        const double beta64 = D.st->beta;
        const bool odd = (D.st->cycle & 1u) != 0u;
        const float* Pold = odd ? F.P2 : F.P;
        float* Pnew = odd ? F.P : F.P2;
        const Lvl& L0 = F.L[0];
        const uint32_t na = w.activeCount();
        const uint32_t wid = g * 4u + (threadIdx.x >> 6);
        const bool valid = wid < na;
        // cgDirection's p of liquid cell k
        auto dir = [&](uint32_t k) {
            const float z = L0.px[k];
            return f64 ? (float)((double)z + beta64 * (double)Pold[k]) : z + beta * Pold[k];
        };
        float vx = 0.0f;
        double ex = 0.0;
        if (valid) {
            I2 c = tileCell(w, wid);
            if (w.inWorld(c)) {
                uint32_t i = w.cellIndex(c);
                float p = 0.0f, q = 0.0f;
                // the cell's and its neighbours' words loaded beside the
                // density (neighbour indices clamp onto the cell), not after
                const float rho = L0.rho[i];
                const uint8_t m = F.fmask[i];
                const float b[4] = {L0.b0[i], L0.b1[i], L0.b2[i], L0.b3[i]};
                const float dgp = L0.diag[i] + F.pin[i];
                const float pi = dir(i);
                float pn[4];
#pragma unroll
                for (int d = 0; d < 4; d++) pn[d] = dir(nbr(i, c.x, c.y, D.W, D.H, d));
                if (rho > 0.0f) {
                    p = pi;
                    float sum = 0.0f;
#pragma unroll
                    for (int d = 0; d < 4; d++)
                        if (m & (1u << d)) sum = sum + b[d] * pn[d];
                    q = dgp * p - sum + 0.0f;
                }
                Pnew[i] = p;
                F.Q[i] = q;
                vx = p * q;
                ex = (double)p * (double)q;
            }
        }
        if (f64) tilePut(ex64[par], ex);
        else tilePut(ux[par], vx);
        __syncthreads();
        float tx = 0.0f;
        double dx = 0.0;
        if (f64) dx = tileSum(ex64[par], ex);
        else tx = tileSum(ux[par], vx);
        par ^= 1u;
        if (valid && (threadIdx.x & 63u) == 0u) {
            const uint32_t b = w.blockIndex(w.activeBlock(wid));
            if (f64) {
                F.part64[2u * b] = dx;
                F.part64[2u * b + 1u] = 0.0;
            } else {
                F.part32[2u * b] = tx;
                F.part32[2u * b + 1u] = 0.0f;
            }
        }
        pend_ += min(4u, na - g * 4u);
        if (flushTiles(Bt, g_it, e_it, it, pend_, &D.st->fdone[2], na)) {
            if (f64) {
                double pq = sumBlocks256(w, F.part64, 0, s64);
                if (threadIdx.x == 0) {
                    D.st->pq = pq;
                    D.st->alpha = pq <= 0.0 ? 0.0 : D.st->rz / pq;
                }
            } else {
                float pq = sumBlocks256(w, F.part32, 0, sx);
                if (threadIdx.x == 0) {
                    D.st->pq32 = pq;
                    D.st->alpha32 = pq <= 0.0f ? 0.0f : D.st->rz32 / pq;
                }
            }
        }
    }
}

// cgUpdate (fluid.wgsl:2852-2880), the tolerance form's norm, and the loop's
// condition: a world iterates again unless its solve has converged
// (converged, fluid.wgsl:2223-2226) or max_cycles are done; the loop runs on
// while any world does.
template <bool ONE>
__global__ void __launch_bounds__(256) k_fUpdate(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    __shared__ uint32_t umost[2][4];  // the upper warps' largest |r| (bits of a non-negative float)
    __shared__ uint32_t runMost;      // the largest |r| of the current world's run
    __shared__ double s64[256];
    __shared__ double ur2[2][128];
    if (threadIdx.x == 0) runMost = 0u;
    uint32_t pend_ = 0;  // tiles finished of the current world, not yet counted
    uint32_t par = 0;    // the tree buffers of this item
    FOR_ITEMS(Bt, L_ACT4, it) {
        FAST_ITEM(Bt, it, D, F, w, g);
        if (D.st->cont == 0u) continue;
        const uint32_t cycle = D.st->cycle;
        const bool f64 = D.st->f64 != 0u, tol = D.st->tol_mode != 0u;
        const float alpha = D.st->alpha32;
        const double alpha64 = D.st->alpha;
        const Lvl& L0 = F.L[0];
        const uint32_t na = w.activeCount();
        const uint32_t wid = g * 4u + (threadIdx.x >> 6);
        const bool valid = wid < na;
        uint32_t m = 0u;
        double r2 = 0.0;
        if (valid) {
            I2 c = tileCell(w, wid);
            if (w.inWorld(c)) {
                uint32_t i = w.cellIndex(c);
                // loaded beside the density, not after it
                const float rho = L0.rho[i], vx = F.X[i], vy = F.R[i], vz = ((cycle & 1u) ? F.P : F.P2)[i];
                const float vw = F.Q[i], py = L0.py[i];
                if (rho > 0.0f) {
                    float r, x;
                    if (f64) {
                        r = (float)((double)vy - alpha64 * (double)vw);
                        x = (float)((double)vx + alpha64 * (double)vz);
                    } else {
                        r = vy - alpha * vw;
                        x = vx + alpha * vz;
                    }
                    F.X[i] = x;
                    F.R[i] = r;
                    L0.px[i] = 0.0f;
                    L0.rx[i] = -r;
                    F.rimx[i] = 0.0f;
                    F.rimy[i] = py;
                    m = __float_as_uint(fabsf(r));
                    r2 = (double)r * (double)r;
                }
            }
        }
        // the tile's largest |r| (a max: any order) and its tree of r^2
        m = __reduce_max_sync(0xffffffffu, m);
        if ((threadIdx.x & 63u) == 32u) umost[par][threadIdx.x >> 6] = m;
        if (tol) tilePut(ur2[par], r2);
        __syncthreads();
        double t2 = 0.0;
        if (tol) t2 = tileSum(ur2[par], r2);
        if (valid && (threadIdx.x & 63u) == 0u) {
            if (tol) D.norm64[2u * w.blockIndex(w.activeBlock(wid))] = t2;
            atomicMax(&runMost, max(m, umost[par][threadIdx.x >> 6]));
        }
        par ^= 1u;
        pend_ += min(4u, na - g * 4u);
        if (worldRunEnds(Bt, L_ACT4, g_it, e_it, it)) {
            // the run's largest |r| into the world's residual slot (a max of
            // maxima: the same word), before its tiles are counted
            __syncthreads();
            if (threadIdx.x == 0) {
                atomicMax(&D.blocks[w.countSlot(COUNT_RESIDUAL + cycle % 3u)], runMost);
                runMost = 0u;
                __threadfence();
            }
        }
        if (flushTiles(Bt, g_it, e_it, it, pend_, &D.st->fdone[3], na)) {
            bool conv;
            if (tol) {
                double rr = sumBlocks256(w, D.norm64, 0, s64);
                double rel = D.st->bnorm2 > 0.0 ? sqrt(rr / D.st->bnorm2) : 0.0;
                if (threadIdx.x == 0) D.st->rel = rel;
                conv = rel <= D.st->tol;
            } else {
                conv = __uint_as_float(__ldcg(&D.blocks[w.countSlot(COUNT_RESIDUAL + cycle % 3u)])) < LIQUID_TOLERANCE;
            }
            if (threadIdx.x == 0) {
                const uint32_t next = cycle + 1u;
                // the mixed form checks the true residual every 8th iteration
                // and before it stops (k_fTrueCheck may then go on)
                const bool check = Bt.mixed != 0u && tol && (conv || (next % 8u) == 0u || next >= Bt.max_cycles);
                const uint32_t cont = (!conv && next < Bt.max_cycles) ? 1u : 0u;
                D.st->cycle = next;
                D.st->cont = cont;
                D.st->check = check ? 1u : 0u;
                if (check && Bt.cond_check) cudaGraphSetConditional(Bt.cond_check, 1u);
                if (cont) {
                    *Bt.loop = 1u;
                    if (Bt.cond) cudaGraphSetConditional(Bt.cond, 1u);
                }
            }
        }
    }
}

// The true residual -(b + A x) of liquid cell i at c, worked in FP64 from the
// FP32 solution, and (floor2) the square of the FP32 rounding of A x there:
// u (|d x| + sum |beta x_n|), u = 2^-24 (the CG's own residual cannot stay
// below that floor's norm).
__device__ __forceinline__ double trueResidualAt(const Dev& D, const FastW& F, I2 c, uint32_t i, double* floor2) {
    const Lvl& L0 = F.L[0];
    const uint8_t m = F.fmask[i];
    const float bb[4] = {L0.b0[i], L0.b1[i], L0.b2[i], L0.b3[i]};
    const double dx = (double)(L0.diag[i] + F.pin[i]) * (double)F.X[i];
    double ax = dx, mag = fabs(dx);
#pragma unroll
    for (int d = 0; d < 4; d++)
        if (m & (1u << d)) {
            const double t = (double)bb[d] * (double)F.X[nbr(i, c.x, c.y, D.W, D.H, d)];
            ax = ax - t;
            mag = mag + fabs(t);
        }
    const double f = mag * 5.9604644775390625e-8;
    *floor2 = f * f;
    return -((double)D.field[8u * (size_t)i + 1u] + ax);
}

// The mixed form's guard, over the worlds k_fUpdate flagged: the FP64 norm
// of the true residual and of the FP32 rounding floor; when the true one
// has drifted above twice the recursive one plus four floors (the
// low-precision preconditioner's rounding lost the recursion's accuracy),
// the world goes on with the true residual put in (k_fTrueFix), else it
// stops or goes on as k_fUpdate decided.
template <bool ONE>
__global__ void __launch_bounds__(256) k_fTrueCheck(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    __shared__ double s64[256], s64b[256];
    uint32_t pend_ = 0;
    FOR_ITEMS(Bt, L_ACT4, it) {
        FAST_ITEM(Bt, it, D, F, w, g);
        if (D.st->check == 0u) continue;
        const Lvl& L0 = F.L[0];
        const uint32_t na = w.activeCount();
        const uint32_t wid = g * 4u + (threadIdx.x >> 6);
        const bool valid = wid < na;
        double r2 = 0.0, f2 = 0.0;
        if (valid) {
            I2 c = tileCell(w, wid);
            if (w.inWorld(c)) {
                const uint32_t i = w.cellIndex(c);
                if (L0.rho[i] > 0.0f) {
                    const double r = trueResidualAt(D, F, c, i, &f2);
                    r2 = r * r;
                }
            }
        }
        const double t2 = tree64x4(s64, r2);
        const double u2 = tree64x4(s64, f2);
        if (valid && (threadIdx.x & 63u) == 0u) {
            const uint32_t b = w.blockIndex(w.activeBlock(wid));
            D.norm64[2u * b] = t2;
            D.norm64[2u * b + 1u] = u2;
        }
        pend_ += min(4u, na - g * 4u);
        if (flushTiles(Bt, g_it, e_it, it, pend_, &D.st->fdone[4], na)) {
            double rr, ff;
            sumBlocks256x2(w, D.norm64, s64, s64b, &rr, &ff);
            if (threadIdx.x == 0) {
                const double bn = D.st->bnorm2;
                const double rel = bn > 0.0 ? sqrt(rr / bn) : 0.0, flo = bn > 0.0 ? sqrt(ff / bn) : 0.0;
                D.st->rel_true = rel;
                D.st->check = 0u;
                if (rel > 2.0 * D.st->rel + 4.0 * flo) {
                    D.st->drift = 1u;
                    if (Bt.cond_drift) cudaGraphSetConditional(Bt.cond_drift, 1u);
                    const uint32_t cont = D.st->cycle < Bt.max_cycles ? 1u : 0u;
                    D.st->cont = cont;
                    if (cont) {
                        *Bt.loop = 1u;
                        if (Bt.cond) cudaGraphSetConditional(Bt.cond, 1u);
                    }
                }
            }
        }
    }
}

// The true residual put in for the recursive one (CG's r and the
// smoother's -r), for the worlds k_fTrueCheck found drifted.
template <bool ONE>
__global__ void k_fTrueFix(Batch Bt, const __grid_constant__ WorldSrc<ONE> src) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    FOR_ITEMS(Bt, L_ACT, it) {
        FAST_ITEM(Bt, it, D, F, w, wid);
        if (D.st->drift == 0u) continue;
        const Lvl& L0 = F.L[0];
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        const uint32_t i = w.cellIndex(c);
        if (L0.rho[i] <= 0.0f) continue;
        double f2;
        const float rf = (float)trueResidualAt(D, F, c, i, &f2);
        F.R[i] = rf;
        L0.rx[i] = -rf;
    }
}

// An iteration's start: the loop stops unless a world's k_fUpdate says
// otherwise; each world still iterating (all of them on the first
// iteration) clears its next residual slot and counts the iteration
// (cgUpdate's first lines, fluid.wgsl:2852-2856), and one with no block
// worked on stops there, as cgUpdate's converged test stops it.
__global__ void k_fLoopStart(Batch Bt) {
    if (threadIdx.x != 0) return;
    if (blockIdx.x == 0) {
        *Bt.loop = 0u;
        if (Bt.cond) cudaGraphSetConditional(Bt.cond, 0u);
        if (Bt.cond_check) cudaGraphSetConditional(Bt.cond_check, 0u);
        if (Bt.cond_drift) cudaGraphSetConditional(Bt.cond_drift, 0u);
    }
    FOR_ITEMS(Bt, L_ONE, it) {
        ITEM_WORLD(Bt, it, D, w, unused_);
        (void)unused_;
        StepState* st = D.st;
        st->drift = 0u;
        if (st->cycle == 0u) st->cont = 1u;
        if (st->cont == 0u) continue;
        const uint32_t cycle = st->cycle;
        D.blocks[w.countSlot(COUNT_RESIDUAL + (cycle + 1u) % 3u)] = 0u;
        D.blocks[w.countSlot(COUNT_CYCLES)] += 1u;
        if (w.activeCount() == 0u) {
            st->cycle = cycle + 1u;
            st->cont = 0u;
        }
    }
}

// cgFinish (fluid.wgsl:2884-2893) and the solve's values back into the
// reference's buffers: field's pressure, divergence left (-r) and drift
// potential, cg's (x, r, p, Ap); and the residual slots the converged
// iterations the reference still dispatches would clear (cgUpdate's first
// lines run whether or not the iteration is skipped).
template <bool ONE>
__global__ void k_fFinish(Batch Bt, const __grid_constant__ WorldSrc<ONE> src, int two_p) {
    __shared__ WorldCopy wc_;
    if (!ONE) worldCopyInit(wc_);
    if (threadIdx.x == 0) {
        FOR_ITEMS(Bt, L_ONE, ot) {
            ITEM_WORLD(Bt, ot, D, w, unused_);
            (void)unused_;
            for (uint32_t c = D.st->cycle; c < Bt.max_cycles; c++)
                D.blocks[w.countSlot(COUNT_RESIDUAL + (c + 1u) % 3u)] = 0u;
        }
    }
    FOR_ITEMS(Bt, L_ACT, it) {
        FAST_ITEM(Bt, it, D, F, w, wid);
        const Lvl& L0 = F.L[0];
        I2 c = lidCell(w, wid);
        if (!w.inWorld(c)) continue;
        uint32_t i = w.cellIndex(c);
        float* f = w.fv(2u * i);
        f[0] = F.X[i];
        if (L0.rho[i] > 0.0f) f[1] = L0.rx[i];
        w.fv(2u * i + 1u)[0] = L0.py[i];
        // the last iteration's p: P2 after an odd number of iterations
        const float* P = (two_p && (D.st->cycle & 1u)) ? F.P2 : F.P;
        reinterpret_cast<float4*>(D.cg)[i] = make_float4(F.X[i], F.R[i], P[i], F.Q[i]);
        *w.gwp(i, G_REGION) = 0u;
    }
}


// ================================================================ the persistent solve
//
// All the iterations of a step's solve in one cooperative launch: each
// reference pass of an iteration is a phase, every CTA taking its share of
// the phase's cells or tiles, the phases separated by a grid barrier; the
// levels of at most 1024 cells are CTA 0's, in its shared memory; the block
// sums are finished by CTA 0 after the barrier.  Same cells, same values,
// same order of every sum as the passes.

// A grid barrier (all CTAs are resident: cooperative launch).  Each wait is
// bounded: past g_spin_limit polls it records ERR_BARRIER and every CTA
// returns false from here on.
__device__ bool gridBarrier(StepState* st, uint32_t nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t* gen = &st->bar_gen;
        const uint32_t g0 = *gen;
        __threadfence();
        const uint32_t arrived = atomicAdd(&st->bar_count, 1u) + 1u;
        int ok = 1;
        if (arrived == nblocks) {
            atomicExch(&st->bar_count, 0u);
            __threadfence();
            atomicAdd(&st->bar_gen, 1u);
        } else {
            uint32_t it = 0;
            const uint32_t limit = g_spin_limit;
            while (*gen == g0) {
                if (++it > limit) {
                    atomicOr(&st->err, ERR_BARRIER);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if ((vld(&st->err) & ERR_BARRIER) != 0u) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// relaxTile (fluid.wgsl:2109-2182), four tiles a 256-thread CTA.
__device__ void relaxGroups(const Fast& F, const W& w, int shift, float (*tpx)[RIM * RIM], float (*tpy)[RIM * RIM],
                            int* s_live, int* s_ox, int* s_oy) {
    const Dev& D = F.D;
    const Lvl& L0 = F.L[0];
    const uint32_t na = w.activeCount();
    const uint32_t total = na + (shift ? D.edge_tiles : 0u);
    const int q = (int)(threadIdx.x >> 6), lane = (int)(threadIdx.x & 63u);
    for (uint32_t g = blockIdx.x; g * 4u < total; g += gridDim.x) {
        const uint32_t j = g * 4u + (uint32_t)q;
        if (lane == 0) {
            int live = 0, ox = 0, oy = 0;
            if (j < total) {
                uint32_t wid = j < na ? j : D.B + (j - na);
                I2 b = tileBlockF(w, wid, shift);
                ox = b.x * BLOCK - shift;
                oy = b.y * BLOCK - shift;
                if (b.x >= 0 && ox < D.W && oy < D.H)
                    live = (int)(w.statesOf(I2{ox / BLOCK, oy / BLOCK}, I2{(ox + BLOCK - 1) / BLOCK, (oy + BLOCK - 1) / BLOCK}) & HAS_FLUID);
            }
            s_live[q] = live;
            s_ox[q] = ox;
            s_oy[q] = oy;
        }
        __syncthreads();
        const bool live = s_live[q] != 0;
        const int ox = s_ox[q], oy = s_oy[q];
        if (live) {
            for (int k = lane; k < RIM * RIM; k += 64) {
                I2 c{ox - 1 + k % RIM, oy - 1 + k / RIM};
                float px = 0.0f, py = 0.0f;
                if (w.inWorld(c)) {
                    uint32_t i = w.cellIndex(c);
                    if (__ldcg(&L0.rho[i]) > 0.0f) {
                        px = __ldcg(&F.rimx[i]);
                        py = __ldcg(&F.rimy[i]);
                    } else {
                        px = __ldcg(&L0.px[i]);
                        py = __ldcg(&L0.py[i]);
                    }
                }
                tpx[q][k] = px;
                tpy[q][k] = py;
            }
        }
        __syncthreads();
        const int lx = lane & 7, ly = lane >> 3;
        const I2 me{ox + lx, oy + ly};
        const int t = (ly + 1) * RIM + lx + 1;
        float rx = 0.0f, ry = 0.0f, bx = 0.0f, by = 0.0f, bz = 0.0f, bw = 0.0f, diag = 0.0f, pinv = 0.0f;
        uint32_t idx = 0;
        bool fluid = false;
        if (live && w.inWorld(me)) {
            idx = w.cellIndex(me);
            fluid = __ldcg(&L0.rho[idx]) > 0.0f;
        }
        if (fluid) {
            rx = __ldcg(&L0.rx[idx]);
            ry = __ldcg(&L0.ry[idx]);
            bx = L0.b0[idx];
            by = L0.b1[idx];
            bz = L0.b2[idx];
            bw = L0.b3[idx];
            diag = L0.diag[idx];
            pinv = F.pin[idx];
        }
        const float dx = diag + pinv, dy = fmaxf(diag, 1e-30f);
        const bool solving = fluid && dx > 0.0f;
        const int color = (me.x + me.y) & 1;
        for (int sw = 0; sw < 2 * SWEEPS; sw++) {
            if (solving && color == (sw & 1)) {
                float sx = bx * tpx[q][t - 1] + by * tpx[q][t + 1] + bz * tpx[q][t - RIM] + bw * tpx[q][t + RIM];
                float sy = bx * tpy[q][t - 1] + by * tpy[q][t + 1] + bz * tpy[q][t - RIM] + bw * tpy[q][t + RIM];
                float nx = mixf(tpx[q][t], (sx - rx) / dx, SMOOTH_OMEGA);
                float ny = mixf(tpy[q][t], (sy - ry) / dy, SMOOTH_OMEGA);
                tpx[q][t] = nx;
                if (diag > 0.0f) tpy[q][t] = ny;
            }
            __syncthreads();
        }
        if (solving) {
            L0.px[idx] = tpx[q][t];
            L0.py[idx] = tpy[q][t];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256, 4) k_fSolve(Fast F, int shifted) {
    extern __shared__ float sm_coarse[];
    __shared__ float tpx[4][RIM * RIM], tpy[4][RIM * RIM];
    __shared__ int s_live[4], s_ox[4], s_oy[4];
    __shared__ float sx[256], sy[256];
    __shared__ double s64[256];
    __shared__ uint32_t most[4];
    __shared__ uint32_t s_off[WIG_MG_LEVELS + 1];
    const Dev& D = F.D;
    W w(D);
    StepState* st = D.st;
    const uint32_t nb = gridDim.x;
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
    const bool f64 = st->f64 != 0u, tol = st->tol_mode != 0u;
    const uint32_t na = w.activeCount();
    const uint32_t lp = F.lp;
    const Lvl& L0 = F.L[0];
    if (na == 0u) {
        // nothing to solve: the first iteration counted, as cgUpdate counts it
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            D.blocks[w.countSlot(COUNT_RESIDUAL + 1u)] = 0u;
            D.blocks[w.countSlot(COUNT_CYCLES)] += 1u;
            st->cycle = 1u;
            st->cont = 0u;
        }
        return;
    }
    for (uint32_t cycle = 0; cycle < F.max_cycles; cycle++) {
        // relax (relaxRims's snapshot is the scratch's rims)
        relaxGroups(F, w, shifted ? BLOCK / 2 : 0, tpx, tpy, s_live, s_ox, s_oy);
        if (!gridBarrier(st, nb)) return;
        for (uint32_t l = 1; l < lp; l++) {
            const uint32_t n = D.level_w[l] * D.level_h[l];
            for (uint32_t j = gt; j < n; j += gn) restrictCell(F.D, F, w, l, j);
            if (!gridBarrier(st, nb)) return;
            for (int color = 0; color < 2; color++) {
                for (uint32_t j = gt; j < n; j += gn) smoothCell(F.D, F, l, color, cycle == 0u, j);
                if (!gridBarrier(st, nb)) return;
            }
        }
        {
            const uint32_t n = D.level_w[lp] * D.level_h[lp];
            for (uint32_t j = gt; j < n; j += gn) restrictCell(F.D, F, w, lp, j);
            if (!gridBarrier(st, nb)) return;
        }
        if (blockIdx.x == 0) coarseLevels(F.D, F, w, lp, sm_coarse, s_off, false);
        if (!gridBarrier(st, nb)) return;
        for (uint32_t l = lp - 1; l >= 1; l--) {
            const uint32_t n = D.level_w[l] * D.level_h[l];
            for (uint32_t j = gt; j < n; j += gn) prolongCell(F.D, F, l, j);
            if (!gridBarrier(st, nb)) return;
            for (int color = 0; color < 2; color++) {
                for (uint32_t j = gt; j < n; j += gn) smoothCell(F.D, F, l, color, false, j);
                if (!gridBarrier(st, nb)) return;
            }
        }
        // prolongFine, and the rims of the relaxation after
        for (uint32_t t = gt; t < na * 64u; t += gn) {
            const uint32_t wid = t >> 6, lane = t & 63u;
            I2 b = w.activeBlock(wid);
            I2 c{b.x * BLOCK + (int)(lane & 7u), b.y * BLOCK + (int)(lane >> 3)};
            if (!w.inWorld(c)) continue;
            uint32_t i = w.cellIndex(c);
            if (L0.rho[i] > 0.0f) {
                const Lvl& U = F.L[1];
                V2 e = prolongedFrom(U.rho, U.px, U.py, (int)D.level_w[1], (int)D.level_h[1], c.x, c.y);
                float px = L0.px[i] + e.x, py = L0.py[i] + e.y;
                L0.px[i] = px;
                L0.py[i] = py;
                F.rimx[i] = px;
                F.rimy[i] = py;
            }
        }
        if (!gridBarrier(st, nb)) return;
        relaxGroups(F, w, shifted ? 0 : BLOCK / 2, tpx, tpy, s_live, s_ox, s_oy);
        if (!gridBarrier(st, nb)) return;
        // cgRho
        for (uint32_t g = blockIdx.x; g * 4u < na; g += gridDim.x) {
            const uint32_t wid = g * 4u + (threadIdx.x >> 6);
            const bool valid = wid < na;
            float vx = 0.0f, vy = 0.0f;
            double ex = 0.0, ey = 0.0;
            if (valid) {
                I2 c = tileCell(w, wid);
                if (w.inWorld(c)) {
                    uint32_t i = w.cellIndex(c);
                    if (L0.rho[i] > 0.0f) {
                        float z = L0.px[i];
                        float r = F.R[i], q = F.Q[i];
                        vx = r * z;
                        vy = q * z;
                        ex = (double)r * (double)z;
                        ey = (double)q * (double)z;
                    }
                }
            }
            float tx = tree64x4(sx, vx);
            float ty = tree64x4(sy, vy);
            double dx = 0.0, dy = 0.0;
            if (f64) {
                dx = tree64x4(s64, ex);
                dy = tree64x4(s64, ey);
            }
            if (valid && (threadIdx.x & 63u) == 0u) {
                const uint32_t b = w.blockIndex(w.activeBlock(wid));
                F.part32[2u * b] = tx;
                F.part32[2u * b + 1u] = ty;
                if (f64) {
                    F.part64[2u * b] = dx;
                    F.part64[2u * b + 1u] = dy;
                }
            }
        }
        if (!gridBarrier(st, nb)) return;
        // cgBeta
        if (blockIdx.x == 0) {
            if (f64) {
                double rz = sumBlocks256(w, F.part64, 0, s64);
                double zq = sumBlocks256(w, F.part64, 1, s64);
                if (threadIdx.x == 0) {
                    double pq = vldd(&st->pq);
                    st->rz = rz;
                    st->beta = (cycle == 0u || pq <= 0.0) ? 0.0 : -zq / pq;
                }
            } else {
                float rz = sumBlocks256(w, F.part32, 0, sx);
                float zq = sumBlocks256(w, F.part32, 1, sx);
                if (threadIdx.x == 0) {
                    float pq = vldf(&st->pq32);
                    st->rz32 = rz;
                    st->beta32 = (cycle == 0u || pq <= 0.0f) ? 0.0f : -zq / pq;
                }
            }
        }
        if (!gridBarrier(st, nb)) return;
        // cgDirection
        {
            const float beta = vldf(&st->beta32);
            const double beta64 = vldd(&st->beta);
            for (uint32_t t = gt; t < na * 64u; t += gn) {
                const uint32_t wid = t >> 6, lane = t & 63u;
                I2 b = w.activeBlock(wid);
                I2 c{b.x * BLOCK + (int)(lane & 7u), b.y * BLOCK + (int)(lane >> 3)};
                if (!w.inWorld(c)) continue;
                uint32_t i = w.cellIndex(c);
                float p = 0.0f;
                if (L0.rho[i] > 0.0f) {
                    float z = L0.px[i];
                    p = f64 ? (float)((double)z + beta64 * (double)F.P[i]) : z + beta * F.P[i];
                }
                F.P[i] = p;
            }
        }
        if (!gridBarrier(st, nb)) return;
        // cgApply
        for (uint32_t g = blockIdx.x; g * 4u < na; g += gridDim.x) {
            const uint32_t wid = g * 4u + (threadIdx.x >> 6);
            const bool valid = wid < na;
            float vx = 0.0f;
            double ex = 0.0;
            if (valid) {
                I2 c = tileCell(w, wid);
                if (w.inWorld(c)) {
                    uint32_t i = w.cellIndex(c);
                    float q = 0.0f;
                    const float p = __ldcg(&F.P[i]);
                    if (L0.rho[i] > 0.0f) {
                        const uint8_t m = F.fmask[i];
                        const float bb[4] = {L0.b0[i], L0.b1[i], L0.b2[i], L0.b3[i]};
                        float sum = 0.0f;
#pragma unroll
                        for (int d = 0; d < 4; d++)
                            if (m & (1u << d)) sum = sum + bb[d] * __ldcg(&F.P[nbr(i, c.x, c.y, D.W, D.H, d)]);
                        float dg = L0.diag[i] + F.pin[i];
                        q = dg * p - sum + 0.0f;
                    }
                    F.Q[i] = q;
                    vx = p * q;
                    ex = (double)p * (double)q;
                }
            }
            float tx = tree64x4(sx, vx);
            double dx = 0.0;
            if (f64) dx = tree64x4(s64, ex);
            if (valid && (threadIdx.x & 63u) == 0u) {
                const uint32_t b = w.blockIndex(w.activeBlock(wid));
                F.part32[2u * b] = tx;
                F.part32[2u * b + 1u] = 0.0f;
                if (f64) {
                    F.part64[2u * b] = dx;
                    F.part64[2u * b + 1u] = 0.0;
                }
            }
        }
        if (!gridBarrier(st, nb)) return;
        // cgAlpha
        if (blockIdx.x == 0) {
            if (f64) {
                double pq = sumBlocks256(w, F.part64, 0, s64);
                if (threadIdx.x == 0) {
                    st->pq = pq;
                    st->alpha = pq <= 0.0 ? 0.0 : vldd(&st->rz) / pq;
                }
            } else {
                float pq = sumBlocks256(w, F.part32, 0, sx);
                if (threadIdx.x == 0) {
                    st->pq32 = pq;
                    st->alpha32 = pq <= 0.0f ? 0.0f : vldf(&st->rz32) / pq;
                }
            }
        }
        if (!gridBarrier(st, nb)) return;
        // cgUpdate (its first lines: the next slot cleared, the iteration counted)
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            D.blocks[w.countSlot(COUNT_RESIDUAL + (cycle + 1u) % 3u)] = 0u;
            D.blocks[w.countSlot(COUNT_CYCLES)] += 1u;
        }
        {
            const float alpha = vldf(&st->alpha32);
            const double alpha64 = vldd(&st->alpha);
            for (uint32_t g = blockIdx.x; g * 4u < na; g += gridDim.x) {
                const uint32_t wid = g * 4u + (threadIdx.x >> 6);
                const bool valid = wid < na;
                if ((threadIdx.x & 63u) == 0u) most[threadIdx.x >> 6] = 0u;
                __syncthreads();
                double r2 = 0.0;
                if (valid) {
                    I2 c = tileCell(w, wid);
                    if (w.inWorld(c)) {
                        uint32_t i = w.cellIndex(c);
                        if (L0.rho[i] > 0.0f) {
                            float vx = F.X[i], vy = F.R[i], vz = __ldcg(&F.P[i]), vw = __ldcg(&F.Q[i]);
                            float r, x;
                            if (f64) {
                                r = (float)((double)vy - alpha64 * (double)vw);
                                x = (float)((double)vx + alpha64 * (double)vz);
                            } else {
                                r = vy - alpha * vw;
                                x = vx + alpha * vz;
                            }
                            F.X[i] = x;
                            F.R[i] = r;
                            L0.px[i] = 0.0f;
                            L0.rx[i] = -r;
                            F.rimx[i] = 0.0f;
                            F.rimy[i] = __ldcg(&L0.py[i]);
                            atomicMax(&most[threadIdx.x >> 6], __float_as_uint(fabsf(r)));
                            r2 = (double)r * (double)r;
                        }
                    }
                }
                double t2 = 0.0;
                if (tol) t2 = tree64x4(s64, r2);
                __syncthreads();
                if (valid && (threadIdx.x & 63u) == 0u) {
                    if (tol) D.norm64[2u * w.blockIndex(w.activeBlock(wid))] = t2;
                    atomicMax(&D.blocks[w.countSlot(COUNT_RESIDUAL + cycle % 3u)], most[threadIdx.x >> 6]);
                }
                __syncthreads();
            }
        }
        if (!gridBarrier(st, nb)) return;
        // converged (fluid.wgsl:2223-2226) for the next iteration
        if (blockIdx.x == 0) {
            bool conv;
            if (tol) {
                double rr = sumBlocks256(w, D.norm64, 0, s64);
                double rel = vldd(&st->bnorm2) > 0.0 ? sqrt(rr / vldd(&st->bnorm2)) : 0.0;
                if (threadIdx.x == 0) st->rel = rel;
                conv = rel <= st->tol;
            } else {
                conv = __uint_as_float(__ldcg(&D.blocks[w.countSlot(COUNT_RESIDUAL + cycle % 3u)])) < LIQUID_TOLERANCE;
            }
            if (threadIdx.x == 0) {
                st->cycle = cycle + 1u;
                st->cont = (!conv && cycle + 1u < F.max_cycles) ? 1u : 0u;
            }
        }
        if (!gridBarrier(st, nb)) return;
        if (vld(&st->cont) == 0u) break;
    }
}

}  // namespace

size_t fast_coarse_smem(const Dev& D, uint32_t lc) {
    size_t n = 0;
    for (uint32_t l = lc; l <= D.levels; l++) n += (size_t)D.level_w[l] * D.level_h[l];
    return SLV_ARRAYS * n * sizeof(float);
}

size_t fast_cluster_smem(const Dev& D, uint32_t lc) {
    if (lc < 1u || lc > D.levels || (size_t)D.level_w[lc] * D.level_h[lc] <= COARSE_CTA_CELLS) return 0;
    return clusterFloats(D.level_w, D.level_h, lc, D.levels, nullptr) * sizeof(float);
}

void fast_zero_level0(const FastW& F, uint32_t cells, cudaStream_t s) { k_fZero<<<148 * 4, 256, 0, s>>>(F, cells); }

void fast_zero_idle(const Batch& Bt, const BatchShape& S, cudaStream_t s) {
    k_fZeroIdle<<<list_grid(S, L_WB, 32), 64, 0, s>>>(Bt);
}

// Launches kernel K's instance for the batch: the single-world one with
// the world as a parameter when `one` is given, else the table one.
#define LAUNCH(K, grid, block, smem, ...)                                                      \
    do {                                                                                       \
        if (one) K<true><<<(grid), (block), (smem), s>>>(Bt, WorldSrc<true>{*one}, ##__VA_ARGS__); \
        else K<false><<<(grid), (block), (smem), s>>>(Bt, WorldSrc<false>{}, ##__VA_ARGS__);       \
    } while (0)
// The same for a kernel over levels stored as T with N threads a CTA.
#define LAUNCH_TN(K, T, N, grid, smem, ...)                                                            \
    do {                                                                                               \
        if (one) K<true, T, N><<<(grid), (N), (smem), s>>>(Bt, WorldSrc<true>{*one}, ##__VA_ARGS__);    \
        else K<false, T, N><<<(grid), (N), (smem), s>>>(Bt, WorldSrc<false>{}, ##__VA_ARGS__);          \
    } while (0)
// The same for a kernel over levels stored as T.
#define LAUNCH_T(K, T, grid, block, smem, ...)                                                        \
    do {                                                                                              \
        if (one) K<true, T><<<(grid), (block), (smem), s>>>(Bt, WorldSrc<true>{*one}, ##__VA_ARGS__);   \
        else K<false, T><<<(grid), (block), (smem), s>>>(Bt, WorldSrc<false>{}, ##__VA_ARGS__);         \
    } while (0)

void fast_setup(const Batch& Bt, const BatchShape& S, const World* one, cudaStream_t s, const Marker* m) {
    if (m) m->fn(m->ctx, WIG_SLOT_F_SETUP, 0);
    LAUNCH(k_fSetup, list_grid(S, L_ACT4, 8), 256, 0);
    if (m) m->fn(m->ctx, WIG_SLOT_F_SETUP, 1);
}

// An IF node at the capture point of stream `outer`, on condition `h`; its
// body captured from `body` (launches on the given stream).
template <class Body>
cudaError_t captureIf(cudaStream_t outer, cudaGraphConditionalHandle h, cudaStream_t inner, Body body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(outer, &cs, nullptr, &g, &deps, &nd);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, deps, nd, &cp);
    if (e != cudaSuccess) return e;
    e = cudaStreamUpdateCaptureDependencies(outer, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return e;
    e = cudaStreamBeginCaptureToGraph(inner, cp.conditional.phGraph_out[0], nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return e;
    body(inner);
    cudaGraph_t captured = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(inner, &captured);
    e = cudaGetLastError();
    return e != cudaSuccess ? e : e2;
}

template <class T>
uint32_t fast_cycle_t(const Batch& Bt0, const BatchShape& S, const World* one, cudaStream_t s, const Marker* m,
                      NestCapture* nest) {
    // the mixed form's check and fix: under IF nodes when captured, with
    // their conditions' handles in the kernels' Batch from the iteration's
    // start (k_fLoopStart clears them, k_fUpdate and k_fTrueCheck set them)
    Batch Bt = Bt0;
    cudaGraphConditionalHandle hc = 0, hd = 0;
    if (Bt.mixed && nest && nest->err == cudaSuccess) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        nest->err = cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr);
        if (nest->err == cudaSuccess) nest->err = cudaGraphConditionalHandleCreate(&hc, g, 0, cudaGraphCondAssignDefault);
        if (nest->err == cudaSuccess) nest->err = cudaGraphConditionalHandleCreate(&hd, g, 0, cudaGraphCondAssignDefault);
        Bt.cond_check = (unsigned long long)hc;
        Bt.cond_drift = (unsigned long long)hd;
    }
    const unsigned G = list_grid(S, L_ACT, 32), G4 = list_grid(S, L_ACT4, S.cg_per_sm);
    const unsigned GR = std::max(std::min((S.max_items[L_RELAX] + 3u) / 4u, 148u * S.relax_per_sm), 1u);
    uint32_t launches = 0;
    auto mark = [&](int slot, int phase) {
        if (m) m->fn(m->ctx, slot, phase);
        if (phase) launches++;
    };
    mark(WIG_SLOT_F_LOOP, 0);
    k_fLoopStart<<<list_grid(S, L_ONE, 1), 32, 0, s>>>(Bt);
    mark(WIG_SLOT_F_LOOP, 1);
    mark(WIG_SLOT_F_RELAX, 0);
    LAUNCH_T(k_fRelax, T, GR, 128, 0, 0);
    mark(WIG_SLOT_F_RELAX, 1);
    // down: each world restricts its levels 1..lc by themselves and smooths
    // those above lc (a kernel a level), then its levels from lc are the
    // coarse kernel's; up: each level above lc prolonged and smoothed
    // a single world's levels of at most two tiles a multiprocessor: 512
    // threads a tile, so each thread takes fewer of its cells in turn
    auto wide = [&](uint32_t list) { return one != nullptr && S.max_items[list] <= 2u * 148u; };
    for (uint32_t l = 1; l <= S.lc_max; l++) {
        mark(WIG_SLOT_F_RESTRICT, 0);
        const uint32_t list = L_RES + l - 1u;
        if (wide(list))
            LAUNCH_TN(k_fDown, T, 512, list_grid(S, list, S.level_per_sm), 0, l);
        else
            LAUNCH_T(k_fDown, T, list_grid(S, list, S.level_per_sm), 256, 0, l);
        mark(WIG_SLOT_F_RESTRICT, 1);
    }
    mark(WIG_SLOT_F_COARSE, 0);
    if (S.cluster && one) {
        // one cluster of CLUSTER_CTAS CTAs
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3(CLUSTER_CTAS);
        c.blockDim = dim3(1024);
        c.dynamicSmemBytes = S.coarse_smem;
        c.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CLUSTER_CTAS;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        c.attrs = at;
        c.numAttrs = 1;
        (void)cudaLaunchKernelEx(&c, k_fCoarseCluster<T>, Bt, WorldSrc<true>{*one});
    } else {
        LAUNCH_T(k_fCoarse, T, list_grid(S, L_ONE, 1), 1024, S.coarse_smem);
    }
    mark(WIG_SLOT_F_COARSE, 1);
    for (uint32_t l = S.lc_max; l >= 1; l--) {
        if (S.max_items[L_SM + l - 1u] == 0u) continue;
        mark(WIG_SLOT_F_PROLONG, 0);
        const uint32_t list = L_SM + l - 1u;
        if (wide(list))
            LAUNCH_TN(k_fUp, T, 512, list_grid(S, list, S.level_per_sm), 0, l);
        else
            LAUNCH_T(k_fUp, T, list_grid(S, list, S.level_per_sm), 256, 0, l);
        mark(WIG_SLOT_F_PROLONG, 1);
    }
    mark(WIG_SLOT_F_PROLONG_FINE, 0);
    LAUNCH_T(k_fProlongFine, T, G, 64, 0);
    mark(WIG_SLOT_F_PROLONG_FINE, 1);
    mark(WIG_SLOT_F_RELAX, 0);
    LAUNCH_T(k_fRelax, T, GR, 128, 0, 1);
    mark(WIG_SLOT_F_RELAX, 1);
    mark(WIG_SLOT_F_RHO_BETA, 0);
    LAUNCH(k_fRhoBeta, G4, 256, 0);
    mark(WIG_SLOT_F_RHO_BETA, 1);
    mark(WIG_SLOT_F_APPLY_ALPHA, 0);
    LAUNCH(k_fApplyAlpha, G4, 256, 0);
    mark(WIG_SLOT_F_APPLY_ALPHA, 1);
    mark(WIG_SLOT_F_UPDATE, 0);
    LAUNCH(k_fUpdate, G4, 256, 0);
    mark(WIG_SLOT_F_UPDATE, 1);
    if (Bt.mixed && hc && hd) {
        // captured: launched only on the iterations that check (not counted
        // among every iteration's launches)
        if (nest->err == cudaSuccess)
            nest->err = captureIf(s, hc, nest->s, [&](cudaStream_t s) { LAUNCH(k_fTrueCheck, G4, 256, 0); });
        if (nest->err == cudaSuccess)
            nest->err = captureIf(s, hd, nest->s, [&](cudaStream_t s) { LAUNCH(k_fTrueFix, G, 64, 0); });
    } else if (Bt.mixed) {
        mark(WIG_SLOT_F_UPDATE, 0);
        LAUNCH(k_fTrueCheck, G4, 256, 0);
        mark(WIG_SLOT_F_UPDATE, 1);
        mark(WIG_SLOT_F_UPDATE, 0);
        LAUNCH(k_fTrueFix, G, 64, 0);
        mark(WIG_SLOT_F_UPDATE, 1);
    }
    return launches;
}

uint32_t fast_cycle(const Batch& Bt, const BatchShape& S, const World* one, cudaStream_t s, const Marker* m,
                    NestCapture* nest) {
    return Bt.mixed ? fast_cycle_t<__half>(Bt, S, one, s, m, nest) : fast_cycle_t<float>(Bt, S, one, s, m, nest);
}

void fast_finish(const Batch& Bt, const BatchShape& S, const World* one, bool two_p, cudaStream_t s, const Marker* m) {
    if (m) m->fn(m->ctx, WIG_SLOT_F_FINISH, 0);
    LAUNCH(k_fFinish, list_grid(S, L_ACT, 32), 64, 0, two_p ? 1 : 0);
    if (m) m->fn(m->ctx, WIG_SLOT_F_FINISH, 1);
}

cudaError_t fast_prepare_attributes(size_t smem) {
    const int b = (int)smem;
    cudaError_t e = cudaFuncSetAttribute(k_fCoarse<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fCoarse<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fCoarse<true, __half>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fCoarse<false, __half>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fCoarseCluster<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fCoarseCluster<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    return e;
}

size_t fast_solve_smem(const Fast& F) { return fast_coarse_smem(F.D, F.lp); }

cudaError_t fast_solve_grid(const Fast& F, uint32_t* grid) {
    int dev = 0, sms = 0, per = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_fSolve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fast_solve_smem(F));
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_fSolve, 256, fast_solve_smem(F));
    if (e != cudaSuccess) return e;
    if (per < 1) return cudaErrorInvalidConfiguration;
    *grid = (uint32_t)(sms * (per < 4 ? per : 4));
    return cudaSuccess;
}

cudaError_t fast_solve(const Fast& F, bool shifted, cudaStream_t s, const Marker* m) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(F.solve_grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = fast_solve_smem(F);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (m) m->fn(m->ctx, WIG_SLOT_F_SOLVE, 0);
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_fSolve, F, shifted ? 1 : 0);
    if (m) m->fn(m->ctx, WIG_SLOT_F_SOLVE, 1);
    return e;
}

}  // namespace wig
