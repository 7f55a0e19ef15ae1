// wig_sched.cu — the work lists of a batch of worlds.
//
// A step of a batch runs each pass as one launch over all the worlds it
// steps: the kernels take items (world, unit of work) from lists that these
// kernels write on the device, so a captured graph serves any subset of the
// batch and any number of blocks worked on.  Each list keeps the worlds in
// the order the host listed them and, within a world, its units in order;
// a world's arithmetic is the same whichever worlds step beside it.
//
// Two points of a step write lists: its start (the worlds' blocks, the
// particles of `sorted`, per-world work, the coarse levels' tiles), and
// after `compact` (the blocks worked on and retired, relaxation tiles, the
// particles of `parts`, whose count syncParticles and syncSeed have set).

#include "wig_sched.cuh"

namespace wig {
namespace {

__device__ __forceinline__ uint32_t cdiv(uint32_t a, uint32_t b) { return (a + b - 1u) / b; }

// The units world k (entry s of the step's subset) has in list L: its
// shape from this step's entry in a pooled batch (the lane's table holds its
// last step's entry until k_schedFill copies this one in, and a world's
// coarse level may have changed since), else from the batch's table.
__device__ uint32_t unitsOf(const Batch& Bt, const SchedCtl& c, uint32_t s, uint32_t L) {
    const World& Wd = c.entries ? c.entries[s] : Bt.worlds[c.sub[s]];
    const Dev& D = Wd.D;
    const bool book = (c.heads ? c.heads[s].book : D.st->book) != 0u;
    // the blocks' counts as compact left them, held to the world's blocks
    // (the lists' room)
    const uint32_t na = min(D.blocks[4u * D.B + COUNT_ACTIVE], D.B);
    const uint32_t nr = min(D.blocks[4u * D.B + COUNT_RETIRED], D.B);
    switch (L) {
    case L_WB: return D.B;
    case L_PS: return book ? 0u : cdiv(min(D.sorted[0], D.cap), 256u);
    case L_ONE_ALL: return 1u;
    case L_ONE: return book ? 0u : 1u;
    case L_PP: return book ? 0u : cdiv(min(D.parts[0], D.cap), 256u);
    case L_ACT: return book ? 0u : na;
    case L_RET: return nr;
    case L_ACT4: return book ? 0u : cdiv(na, 4u);
    case L_RELAX: return book ? 0u : na + D.edge_tiles;
    default: break;
    }
    if (L >= L_RES && L < L_RES + WIG_MG_LEVELS) {
        const uint32_t l = L - L_RES + 1u;
        return (!book && l <= Wd.S.lc && l <= D.levels) ? levelTiles(D.level_w[l], D.level_h[l]) : 0u;
    }
    if (L >= L_SM && L < L_SM + WIG_MG_LEVELS) {
        const uint32_t l = L - L_SM + 1u;
        return (!book && l < Wd.S.lc) ? levelTiles(D.level_w[l], D.level_h[l]) : 0u;
    }
    return 0u;
}

// The lists each point writes.
__constant__ uint32_t kPhaseA[] = {L_WB, L_PS, L_ONE_ALL, L_ONE,
                                   L_RES + 0, L_RES + 1, L_RES + 2, L_RES + 3, L_RES + 4, L_RES + 5, L_RES + 6, L_RES + 7,
                                   L_SM + 0, L_SM + 1, L_SM + 2, L_SM + 3, L_SM + 4, L_SM + 5, L_SM + 6, L_SM + 7};
__constant__ uint32_t kPhaseB[] = {L_ACT, L_RET, L_ACT4, L_RELAX, L_PP};
constexpr uint32_t N_PHASE_A = 20, N_PHASE_B = 5;

// One CTA of 32 warps: warp w scans list w of the phase over the subset
// (32 entries at a time), leaving each entry's first item in off and the
// list's total in count.
__global__ void __launch_bounds__(1024) k_schedScan(Batch Bt, SchedCtl c, int phase) {
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nl = phase == 0 ? N_PHASE_A : N_PHASE_B;
    if (warp >= nl) return;
    const uint32_t L = phase == 0 ? kPhaseA[warp] : kPhaseB[warp];
    const uint32_t n = *c.nsub;
    uint32_t* off = c.off + (size_t)L * (c.max_worlds + 1u);
    uint32_t run = 0;
    for (uint32_t s0 = 0; s0 < n; s0 += 32u) {
        const uint32_t s = s0 + lane;
        const uint32_t u = s < n ? unitsOf(Bt, c, s, L) : 0u;
        uint32_t incl = u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += v;
        }
        if (s < n) off[s] = run + incl - u;
        run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
        off[n] = run;
        c.count[L] = run;
    }
}

// The items: CTA quarter q of entry s writes units q*256 + t, +1024, ...
// At the step's start, also each world's StepState from its head.
__global__ void __launch_bounds__(256) k_schedFill(Batch Bt, SchedCtl c, int phase) {
    const uint32_t n = *c.nsub;
    const uint32_t nl = phase == 0 ? N_PHASE_A : N_PHASE_B;
    const uint32_t lb = Bt.lbits;
    for (uint32_t g = blockIdx.x; g < n * 4u; g += gridDim.x) {
        const uint32_t s = g >> 2, q = g & 3u;
        const uint32_t k = c.sub[s];
        if (phase == 0 && c.heads && q == 0u && threadIdx.x == 0) {
            StepState* st = Bt.worlds[k].D.st;
            const StepHead& h = c.heads[s];
            st->P = h.P;
            st->tol_mode = h.tol_mode;
            st->f64 = h.f64;
            st->book = h.book;
            st->viscous = h.viscous;
            st->shift_first = h.shift_first;
            st->tol = h.tol;
            st->err = 0u;
            st->cycles_run = 0u;
            st->rel = 1.0;
            st->bnorm2 = 0.0;
            st->rz = 0.0; st->pq = 0.0; st->alpha = 0.0; st->beta = 0.0;
            st->cycle = 0u;
            st->cont = 0u;
            for (int f = 0; f < 6; f++) st->fdone[f] = 0u;
            st->check = 0u;
            st->drift = 0u;
            st->rel_true = 0.0;
            st->rz32 = 0.0f; st->pq32 = 0.0f; st->alpha32 = 0.0f; st->beta32 = 0.0f;
            st->bar_count = 0u;
            st->bar_gen = 0u;
        }
        if (phase == 0 && c.entries && q == 0u) {
            // the world's table entry for this step (the scan above read it
            // from the entries)
            const uint4* src = reinterpret_cast<const uint4*>(&c.entries[s]);
            uint4* dst = reinterpret_cast<uint4*>(&c.table[k]);
            for (uint32_t i = threadIdx.x; i < sizeof(World) / 16u; i += blockDim.x) dst[i] = src[i];
        }
        for (uint32_t li = 0; li < nl; li++) {
            const uint32_t L = phase == 0 ? kPhaseA[li] : kPhaseB[li];
            const uint32_t* off = c.off + (size_t)L * (c.max_worlds + 1u);
            const uint32_t first = off[s], units = off[s + 1u] - first;
            uint32_t* out = c.items + Bt.base[L] + first;
            const uint32_t tag = (uint32_t)((uint64_t)k << lb);
            for (uint32_t j = q * 256u + threadIdx.x; j < units; j += 1024u) out[j] = tag | j;
        }
    }
}

}  // namespace

void sched_lists(const Batch& Bt, const SchedCtl& c, const BatchShape& S, int phase, cudaStream_t s) {
    k_schedScan<<<1, 1024, 0, s>>>(Bt, c, phase);
    unsigned g = S.worlds * 4u, cap = 148u * 8u;
    k_schedFill<<<g < cap ? g : cap, 256, 0, s>>>(Bt, c, phase);
}

}  // namespace wig
