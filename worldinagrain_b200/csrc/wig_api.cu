// wig_api.cu — the C ABI (include/wig_fluid.h, include/wig_batch.h): world
// handles and batches, bound buffers, and the step driver that replaces
// Simulation.encodeFluid (js/sim.js:2466-2612).
//
// Every handle is a batch: a table of worlds in device memory and, per step
// lane, the work lists the kernels take their items from.  A single-world
// handle (wig_fluid) is a batch of one.  A step is the reference's pass
// sequence, recorded once per shape (max cycles, flags) into a CUDA graph
// and replayed: the per-step inputs (each world's Params uniform and its
// part of the step) reach the device as one small copy from pinned host
// memory ahead of the graph, and the report words come back as one small
// copy after it, the reference's writeBuffer and mapped report buffer
// (js/sim.js:1975-1995, :1763, :1882-1900).

#include <algorithm>
#include <cmath>
#include <array>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/wig_batch.h"
#include "wig_device.cuh"
#include "wig_fast.cuh"
#include "wig_passes.cuh"
#include "wig_sched.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace

namespace wig {
void set_last_error(const std::string& msg) { g_last_error = msg; }
__device__ uint32_t g_loop_limit = LOOP_LIMIT;
__device__ uint32_t g_spin_limit = BARRIER_SPIN_LIMIT;
}  // namespace wig

namespace {

#define CUDA_TRY(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(WIG_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device-side report of a world: the FLUID_COUNT words, the particle count
// and the solve's residuals, gathered by k_report at the end of a step.
struct Report {
    uint32_t count[WIG_FLUID_STATS];
    uint32_t particles;
    uint32_t err;
    uint32_t short_of_tol;  // a tolerance-form solve of a nonzero b stopped above its tolerance
    uint32_t tried;         // particles the step's sync and seeding put into `parts` (past its room: lost)
    double rel;
    double bnorm2;
    double rel_true;
};

// Each world's report into its slot (by world) and the lane's (by the
// world's place in the step's list).
__global__ void k_report(wig::Batch Bt, Report* by_world, Report* by_entry) {
    if (threadIdx.x != 0) return;
    FOR_ITEMS(Bt, wig::L_ONE_ALL, it) {
        const uint32_t k = (uint32_t)((uint64_t)it >> Bt.lbits);
        const wig::Dev& D = Bt.worlds[k].D;
        Report r;
        for (uint32_t c = 0; c < WIG_FLUID_STATS; c++) r.count[c] = D.blocks[4u * D.B + c];
        r.particles = D.sorted[0];
        r.tried = D.parts[0];
        r.err = D.st->err;
        // a full step of the tolerance form whose solve stopped (max_cycles
        // run) with the residual still above the tolerance
        r.short_of_tol = (D.st->tol_mode && !D.st->book && D.st->bnorm2 > 0.0 && D.st->rel > D.st->tol) ? 1u : 0u;
        r.rel = D.st->rel;
        r.bnorm2 = D.st->bnorm2;
        r.rel_true = D.st->rel_true;
        by_world[k] = r;
        by_entry[g_it] = r;
    }
}

constexpr int RING = 8;

struct Graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    uint32_t outside = 0;  // kernels outside the iteration loop
    uint32_t body = 0;     // kernels of one iteration
};

// A step lane: its work lists, its per-step upload ring, its graphs.
struct Lane {
    uint32_t* d_items = nullptr;
    uint32_t* d_count = nullptr;
    uint32_t* d_off = nullptr;
    uint32_t* d_loop = nullptr;
    char* d_up = nullptr;          // nsub, sub[], heads[]
    char* h_up = nullptr;          // pinned, RING slots
    cudaEvent_t up_ev[RING] = {};
    int up_at = 0;
    Report* d_rsub = nullptr;
    Report* h_rsub = nullptr;      // pinned
    // pooled batches: the lane's own world table and its pool of the
    // per-step memory (each stepping world's borrowed buffers and scratch)
    wig::World* d_table = nullptr;
    char* d_pool = nullptr;
    uint64_t pool_bytes = 0;
    wig::Batch Bt{};
    wig::SchedCtl ctl{};
    wig::BatchShape S{};           // the shape the lane's step records with (step_shape)
    std::map<uint64_t, Graph> graphs;
    cudaStream_t cap = nullptr, cap2 = nullptr, cap3 = nullptr;
    cudaStream_t last_stream = nullptr;
    uint32_t last_launches = 0, last_body = 0;
};

size_t align256(size_t x) { return (x + 255u) & ~(size_t)255u; }

}  // namespace

struct wig_batch {
    uint32_t K = 0;
    uint64_t blocks_all = 0;  // the worlds' blocks, summed
    int device = 0;
    std::vector<wig_world_layout> L;
    std::vector<wig::World> hw;       // host copy of the world table
    wig::World* d_worlds = nullptr;
    wig_elem* d_elems = nullptr;
    wig::StepState* d_st = nullptr;   // K
    Report* d_report = nullptr;       // K
    Report* h_report = nullptr;       // K, pinned
    void* scratch = nullptr;          // the fast form's scratch and FP64 partials of every world
    void* arena = nullptr;            // the worlds' buffers (batches made by wig_batch_create)
    std::vector<void*> wmem;          // each world's allocation (batches made by wig_batch_create_deferred)
    uint64_t resident = 0;            // bytes of the admitted worlds' allocations
    std::vector<std::array<void*, 7>> own;  // buffers a single-world handle allocated at bind
    std::vector<char> bound, dirty;
    std::vector<char> shifted_first;
    std::vector<cudaStream_t> stepped_on;   // the stream of each world's last step
    std::vector<int> stepped_lane;
    wig::BatchShape S{};
    uint32_t lbits = 31;
    uint32_t solve_grid = 0;          // the persistent solve's CTAs (a batch of one world)
    Lane lane[WIG_BATCH_LANES];
    size_t up_bytes = 0;              // one upload slot
    size_t entries_at = 0;            // offset of the staged world entries in a slot (pooled batches)
    bool pooled = false;              // per-step memory from the lanes' pools
};

struct wig_fluid {
    wig_batch* b = nullptr;
};

namespace {

int layout_of(const wig_world_desc* d, wig_world_layout* L) {
    if (!d || !L) return fail(WIG_E_ARG, "null descriptor");
    if (d->width == 0 || d->height == 0 || d->width > 32768 || d->height > 32768)
        return fail(WIG_E_ARG, "world size out of range (1..32768 per side)");
    std::memset(L, 0, sizeof(*L));
    uint64_t W = d->width, H = d->height, C = W * H;
    uint64_t F = (W + 1) * H + W * (H + 1);
    L->width = (uint32_t)W;
    L->height = (uint32_t)H;
    L->liquid_per_cell = d->liquid_per_cell ? d->liquid_per_cell : 4u;
    if (L->liquid_per_cell > 64) return fail(WIG_E_ARG, "liquid_per_cell out of range (1..64)");
    uint64_t cap = d->capacity;
    if (!cap) {
        // ceil(C * ppc * 1.25) exactly (js/sim.js:747)
        uint64_t num = C * L->liquid_per_cell * 5ull;
        cap = (num + 3ull) / 4ull;
    }
    if (cap > 0x3fffffffull) return fail(WIG_E_ARG, "particle capacity too large");
    L->capacity = (uint32_t)cap;
    L->cell_count = (uint32_t)C;
    L->face_count = (uint32_t)F;
    L->blocks_wide = (uint32_t)((W + 7) / 8);
    L->block_count = L->blocks_wide * (uint32_t)((H + 7) / 8);
    L->edge_tiles = (uint32_t)((W + 7) / 8 + (H + 7) / 8 + 1);
    uint64_t levelCells = 0;
    for (uint32_t l = 1; l <= WIG_MG_LEVELS; l++) {
        uint64_t lw = (W + (1ull << l) - 1) >> l, lh = (H + (1ull << l) - 1) >> l;
        L->level_w[l - 1] = (uint32_t)lw;
        L->level_h[l - 1] = (uint32_t)lh;
        L->levels = l;
        levelCells += lw * lh;
        if (lw * lh <= WIG_MG_COARSEST) break;
    }
    if ((uint64_t)L->level_w[L->levels - 1] * L->level_h[L->levels - 1] > WIG_MG_COARSEST)
        return fail(WIG_E_ARG, "world too large for the multigrid's levels");
    L->cells_bytes = 16ull * (C + (C + 1) / 2);
    L->particles_bytes = 16ull + 48ull * L->capacity;
    L->counters_bytes = 4ull * (11ull * C + 2ull * F);
    L->field_bytes = 16ull * ((C + levelCells) * 2ull + F + 2ull * ((F + 3) / 4));
    L->blocks_bytes = 4ull * (5ull * L->block_count + WIG_FLUID_STATS);
    L->cg_bytes = 16ull * (C + L->block_count + 1);
    return WIG_OK;
}

uint64_t buffer_bytes(const wig_world_layout& L, int which) {
    switch (which) {
    case 0: return L.cells_bytes;
    case 1: case 2: return L.particles_bytes;
    case 3: return L.counters_bytes;
    case 4: return L.field_bytes;
    case 5: return L.blocks_bytes;
    case 6: return L.cg_bytes;
    default: return 0;
    }
}

void** buffer_slot(wig::Dev& D, int which) {
    switch (which) {
    case 0: return (void**)&D.cells;
    case 1: return (void**)&D.sorted;
    case 2: return (void**)&D.parts;
    case 3: return (void**)&D.counters;
    case 4: return (void**)&D.field;
    case 5: return (void**)&D.blocks;
    case 6: return (void**)&D.cg;
    default: return nullptr;
    }
}

// The shape fields of a world's descriptor.
void dev_shape(wig::Dev& D, const wig_world_layout& L) {
    D.W = (int)L.width;
    D.H = (int)L.height;
    D.C = L.cell_count;
    D.F = L.face_count;
    D.B = L.block_count;
    D.BW = L.blocks_wide;
    D.bw_mul = 0xffffffffu / L.blocks_wide;
    D.BH = L.block_count / L.blocks_wide;
    D.cap = L.capacity;
    D.ppc = L.liquid_per_cell;
    D.edge_tiles = L.edge_tiles;
    D.levels = L.levels;
    D.level_w[0] = L.width;
    D.level_h[0] = L.height;
    uint32_t at = 2u * D.C + D.F + 2u * ((D.F + 3u) / 4u);
    D.level_start[0] = 0;
    for (uint32_t l = 1; l <= WIG_MG_LEVELS; l++) {
        D.level_w[l] = l <= L.levels ? L.level_w[l - 1] : 0u;
        D.level_h[l] = l <= L.levels ? L.level_h[l - 1] : 0u;
        D.level_start[l] = at;
        at += 2u * D.level_w[l] * D.level_h[l];
    }
}

// Bytes of a world's fast scratch and FP64 partials.
size_t scratch_bytes(const wig::Dev& D) {
    const size_t C = D.C;
    size_t bytes = align256(C) + 18u * align256(C * 4u) + align256(4u * C * 2u);  // + level 0's binary16 copies
    for (uint32_t l = 1; l <= D.levels; l++) {
        bytes += 12u * align256((size_t)D.level_w[l] * D.level_h[l] * 4u);
        bytes += align256(5u * (size_t)D.level_w[l] * D.level_h[l] * 2u);  // the binary16 operator
    }
    bytes += align256(2u * (size_t)D.B * 4u) + 3u * align256(2u * (size_t)D.B * 8u);
    return bytes;
}

// Lays a world's scratch out from p (scratch_bytes of it); the coarse
// kernel from its first level of at most coarse_cells cells.
void scratch_take(wig::World& Wd, char* p, uint32_t coarse_cells) {
    wig::Dev& D = Wd.D;
    wig::FastW& F = Wd.S;
    auto take = [&](size_t n) { char* q = p; p += align256(n); return q; };
    auto fl = [&](size_t n) { return reinterpret_cast<float*>(take(n * 4u)); };
    const size_t C = D.C;
    F.fmask = reinterpret_cast<uint8_t*>(take(C));
    for (uint32_t l = 0; l <= D.levels; l++) {
        const size_t n = l == 0 ? C : (size_t)D.level_w[l] * D.level_h[l];
        wig::Lvl& V = F.L[l];
        V.px = fl(n); V.py = fl(n); V.rx = fl(n); V.ry = fl(n); V.rho = fl(n);
        V.b0 = fl(n); V.b1 = fl(n); V.b2 = fl(n); V.b3 = fl(n); V.diag = fl(n);
        V.ux = l == 0 ? nullptr : fl(n);
        V.uy = l == 0 ? nullptr : fl(n);
    }
    F.H[0] = wig::LvlH{reinterpret_cast<__half*>(take(4u * C * 2u)), (uint32_t)C, 0u};
    for (uint32_t l = 1; l <= D.levels; l++) {
        const size_t n = (size_t)D.level_w[l] * D.level_h[l];
        F.H[l] = wig::LvlH{reinterpret_cast<__half*>(take(5u * n * 2u)), (uint32_t)n, 0u};
    }
    F.pin = fl(C); F.rimx = fl(C); F.rimy = fl(C);
    F.X = fl(C); F.R = fl(C); F.P = fl(C); F.Q = fl(C); F.P2 = fl(C);
    F.part32 = fl(2u * (size_t)D.B);
    F.part64 = reinterpret_cast<double*>(take(2u * (size_t)D.B * 8u));
    D.part64 = reinterpret_cast<double*>(take(2u * (size_t)D.B * 8u));
    D.norm64 = reinterpret_cast<double*>(take(2u * (size_t)D.B * 8u));
    F.lc = wig::coarse_level(D, coarse_cells);
    F.lp = D.levels;
    for (uint32_t l = 1; l <= D.levels; l++)
        if ((size_t)D.level_w[l] * D.level_h[l] <= wig::PERSISTENT_CTA_CELLS) { F.lp = l; break; }
}

uint64_t world_buffers_bytes(const wig_world_layout& L) {
    uint64_t n = 0;
    for (int k = 0; k < 7; k++) n += align256(buffer_bytes(L, k));
    return n;
}

// A pooled world's split: what stays on the device between its steps and
// what a step borrows from its lane's pool.  Borrowed: `parts` (syncParticles
// refills it every step), `cg` (cgStart and the solve's finish write it, no
// pass reads it across steps) and the fast form's scratch (the step zeroes
// it where it is read before written).  Kept: the other buffers, `field`
// without its coarse levels (the fast form keeps those in its scratch).
bool borrowed(int which) { return which == 2 || which == 6; }
uint64_t persistent_buffer_bytes(const wig_world_layout& L, int which) {
    if (borrowed(which)) return 0;
    if (which == 4) {
        const uint64_t F = L.face_count;
        return 16ull * (2ull * L.cell_count + F + 2ull * ((F + 3) / 4));
    }
    return buffer_bytes(L, which);
}
uint64_t persistent_bytes(const wig_world_layout& L) {
    uint64_t n = 0;
    for (int k = 0; k < 7; k++) n += align256(persistent_buffer_bytes(L, k));
    return n;
}
uint64_t transient_bytes(const wig_world_layout& L, const wig::Dev& D) {
    return align256(buffer_bytes(L, 2)) + align256(buffer_bytes(L, 6)) + scratch_bytes(D);
}

uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

void destroy_batch(wig_batch* b);

// Frees a lane's graphs.
void drop_graphs(Lane& ln) {
    for (auto& kv : ln.graphs) {
        if (kv.second.ge) cudaGraphExecDestroy(kv.second.ge);
        if (kv.second.g) cudaGraphDestroy(kv.second.g);
    }
    ln.graphs.clear();
}

int upload_world_entry(wig_batch* b, uint32_t k) {
    CUDA_TRY(cudaMemcpy(b->d_worlds + k, &b->hw[k], sizeof(wig::World), cudaMemcpyHostToDevice));
    return WIG_OK;
}

// The level part of a batch's shape for its coarse_cells: each world's
// coarse level (into its table entry), the level lists' current lengths,
// the deepest level restricted by a tile kernel, the coarse kernel's memory
// (a single world's from a level too large for one CTA: the cluster
// kernel's).
void level_shape(wig_batch* b) {
    wig::BatchShape& S = b->S;
    for (uint32_t l = 0; l < WIG_MG_LEVELS; l++) {
        S.max_items[wig::L_RES + l] = 0;
        S.max_items[wig::L_SM + l] = 0;
    }
    S.lc_max = 0;
    S.coarse_smem = 0;
    S.cluster = 0;
    for (uint32_t k = 0; k < b->K; k++) {
        wig::World& Wd = b->hw[k];
        const wig::Dev& D = Wd.D;
        const uint32_t lc = wig::coarse_level(D, S.coarse_cells);
        Wd.S.lc = lc;
        for (uint32_t l = 1; l <= D.levels; l++) {
            const uint32_t ch = wig::levelTiles(D.level_w[l], D.level_h[l]);
            if (l <= lc) S.max_items[wig::L_RES + l - 1] += ch;
            if (l < lc) S.max_items[wig::L_SM + l - 1] += ch;
        }
        S.lc_max = std::max(S.lc_max, lc);
        const size_t c = b->K == 1 ? wig::fast_cluster_smem(D, lc) : 0;
        if (c) S.cluster = 1;
        S.coarse_smem = std::max(S.coarse_smem, c ? c : wig::fast_coarse_smem(D, lc));
    }
}

// How a batch holds its worlds' device memory: a single world's scratch with
// its buffers bound later (wig_fluid_bind); every world's buffers and
// scratch packed in two allocations; or each world's own allocation, made
// when it is admitted and freed when it is evicted (serving).
enum class Alloc { Single, Packed, Deferred };

// A batch of n worlds with their shapes, lanes and (per `how`) memory.
int make_batch(const wig_world_desc* descs, uint32_t n, const wig_elem* elems, uint32_t n_elems, Alloc how,
               wig_batch** out) {
    if (!out) return fail(WIG_E_ARG, "null output handle");
    *out = nullptr;
    if (!descs || n == 0 || n > WIG_BATCH_MAX_WORLDS) return fail(WIG_E_ARG, "world count out of range");
    if (!elems || n_elems == 0 || n_elems > WIG_MAX_ELEMS) return fail(WIG_E_ARG, "element table empty or too long");
    if (n_elems <= WIG_ELEM_WATER) return fail(WIG_E_ARG, "element table must reach WATER (id 3)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(WIG_E_NO_DEVICE, "no CUDA device");
    }
    wig_batch* b = new (std::nothrow) wig_batch();
    if (!b) return fail(WIG_E_OOM, "host allocation failed");
    auto bail = [&](int code, const std::string& m) {
        std::string keep = m;
        destroy_batch(b);
        return fail(code, keep);
    };
    b->K = n;
    cudaGetDevice(&b->device);
    b->L.resize(n);
    b->hw.assign(n, wig::World{});
    b->own.assign(n, std::array<void*, 7>{});
    b->bound.assign(n, 0);
    b->dirty.assign(n, 1);
    b->shifted_first.assign(n, 0);
    b->stepped_on.assign(n, nullptr);
    b->stepped_lane.assign(n, -1);
    for (uint32_t k = 0; k < n; k++) {
        int rc = layout_of(&descs[k], &b->L[k]);
        if (rc) {
            std::string m = g_last_error;
            destroy_batch(b);
            return fail(rc, "world " + std::to_string(k) + ": " + m);
        }
        dev_shape(b->hw[k].D, b->L[k]);
    }
    // the shape: list sizes, coarse kernel's memory, item bits; the level
    // lists' room for any coarse level (every level above the coarsest)
    wig::BatchShape& S = b->S;
    std::memset(&S, 0, sizeof(S));
    S.worlds = n;
    // a single world's defaults are the shapes measured fastest on the
    // 1024x1024 world in its step graph (coarse kernel from 32x32, 32 CTAs a
    // multiprocessor for the level kernels, 64 for the relaxation: 170.5
    // Mcells/s against 168.8 from 64x64 and 166.8 from 16x16); its CG
    // kernels run fastest with fewer CTAs, each taking more tiles and fewer
    // of them counting into the world's last-tile counter.  A batch's are
    // the autotuner's starting point.
    S.coarse_cells = n == 1 ? 2048u : wig::COARSE_CTA_CELLS;
    S.level_per_sm = n == 1 ? 32u : 8u;
    S.cg_per_sm = n == 1 ? 4u : 8u;
    S.relax_per_sm = n == 1 ? 64u : 16u;
    uint64_t most_units = 1, max_items[wig::L_COUNT] = {0};
    size_t scratch_total = 0;
    for (uint32_t k = 0; k < n; k++) {
        wig::World& Wd = b->hw[k];
        const wig::Dev& D = Wd.D;
        scratch_total += scratch_bytes(D);
        const uint32_t lc = D.levels;
        const uint64_t pch = cdiv(D.cap, 256);
        max_items[wig::L_WB] += D.B;
        max_items[wig::L_PS] += pch;
        max_items[wig::L_PP] += pch;
        max_items[wig::L_ACT] += D.B;
        max_items[wig::L_RET] += D.B;
        max_items[wig::L_ACT4] += cdiv(D.B, 4);
        max_items[wig::L_RELAX] += D.B + D.edge_tiles;
        max_items[wig::L_ONE_ALL] += 1;
        max_items[wig::L_ONE] += 1;
        for (uint32_t l = 1; l <= WIG_MG_LEVELS; l++) {
            const uint64_t ch = l <= D.levels ? wig::levelTiles(D.level_w[l], D.level_h[l]) : 0u;
            if (l <= lc && l <= D.levels) max_items[wig::L_RES + l - 1] += ch;
            if (l < lc) max_items[wig::L_SM + l - 1] += ch;
            if (l <= D.levels) most_units = std::max<uint64_t>(most_units, ch);
        }
        most_units = std::max<uint64_t>(most_units, std::max<uint64_t>(D.B + D.edge_tiles, pch));
        S.levels = std::max(S.levels, D.levels);
    }
    uint32_t bits = 1;
    while (bits < 31 && (1ull << bits) <= most_units) bits++;
    if ((1ull << bits) <= most_units) return bail(WIG_E_ARG, "a world is too large for the work lists");
    if (bits < 31 && (uint64_t)n > (1ull << (32 - bits))) return bail(WIG_E_ARG, "too many worlds of this size in one batch");
    b->lbits = bits;
    uint64_t items_total = 0;
    uint32_t base[wig::L_COUNT];
    for (uint32_t l = 0; l < wig::L_COUNT; l++) {
        if (max_items[l] > 0xffffffffull) return bail(WIG_E_ARG, "work lists too long");
        S.max_items[l] = (uint32_t)max_items[l];
        base[l] = (uint32_t)items_total;
        items_total += max_items[l];
    }
    if (items_total > 0xffffffffull) return bail(WIG_E_ARG, "work lists too long");
    level_shape(b);
    for (uint32_t k = 0; k < n; k++) b->blocks_all += b->hw[k].D.B;
    if (S.coarse_smem > 220u * 1024u) return bail(WIG_E_ARG, "coarse levels too large for one CTA");
    if (wig::fast_prepare_attributes(S.coarse_smem) != cudaSuccess) return bail(WIG_E_CUDA, "cudaFuncSetAttribute");

    // device memory: elements, step states, reports, world table, scratch
    if (cudaMalloc(&b->d_elems, sizeof(wig_elem) * n_elems) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc elems");
    if (cudaMemcpy(b->d_elems, elems, sizeof(wig_elem) * n_elems, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(WIG_E_CUDA, "cudaMemcpy elems");
    if (cudaMalloc(&b->d_st, sizeof(wig::StepState) * n) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc step states");
    cudaMemset(b->d_st, 0, sizeof(wig::StepState) * n);
    if (cudaMalloc(&b->d_report, sizeof(Report) * n) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc reports");
    cudaMemset(b->d_report, 0, sizeof(Report) * n);
    if (cudaMallocHost(&b->h_report, sizeof(Report) * n) != cudaSuccess) return bail(WIG_E_OOM, "cudaMallocHost reports");
    std::memset(b->h_report, 0, sizeof(Report) * n);
    if (cudaMalloc(&b->d_worlds, sizeof(wig::World) * n) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc world table");
    for (uint32_t k = 0; k < n; k++) {
        wig::World& Wd = b->hw[k];
        Wd.D.elems = b->d_elems;
        Wd.D.n_elems = n_elems;
        Wd.D.st = b->d_st + k;
    }
    if (how != Alloc::Deferred) {
        if (cudaMalloc(&b->scratch, scratch_total) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc fast scratch");
        cudaMemset(b->scratch, 0, scratch_total);
        char* p = static_cast<char*>(b->scratch);
        for (uint32_t k = 0; k < n; k++) {
            scratch_take(b->hw[k], p, b->S.coarse_cells);
            p += scratch_bytes(b->hw[k].D);
        }
    } else {
        b->wmem.assign(n, nullptr);
        // stream-ordered allocations that stay with the pool when freed, so
        // admitting a world after an eviction is a pool hit
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, b->device) == cudaSuccess) {
            uint64_t keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (how == Alloc::Packed) {
        uint64_t total = 0;
        for (uint32_t k = 0; k < n; k++) total += world_buffers_bytes(b->L[k]);
        if (cudaMalloc(&b->arena, total) != cudaSuccess) {
            cudaGetLastError();
            return bail(WIG_E_OOM, "cudaMalloc of the worlds' buffers failed");
        }
        if (cudaMemset(b->arena, 0, total) != cudaSuccess) return bail(WIG_E_CUDA, "cudaMemset of the worlds' buffers");
        char* p = static_cast<char*>(b->arena);
        for (uint32_t k = 0; k < n; k++) {
            for (int w = 0; w < 7; w++) {
                *buffer_slot(b->hw[k].D, w) = p;
                p += align256(buffer_bytes(b->L[k], w));
            }
            b->bound[k] = 1;
        }
    }
    if (cudaMemcpy(b->d_worlds, b->hw.data(), sizeof(wig::World) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(WIG_E_CUDA, "cudaMemcpy world table");
    if (n == 1) {
        wig::Fast F0;
        static_cast<wig::FastW&>(F0) = b->hw[0].S;
        F0.D = b->hw[0].D;
        if (wig::fast_solve_grid(F0, &b->solve_grid) != cudaSuccess) return bail(WIG_E_CUDA, "occupancy of the persistent solve");
    }

    // lanes
    b->up_bytes = 8u + ((4u * (size_t)n + 7u) & ~(size_t)7u) + sizeof(wig::StepHead) * n;
    if (how == Alloc::Deferred) {
        // room for the stepping worlds' table entries of a pooled step
        b->entries_at = (b->up_bytes + 15u) & ~(size_t)15u;
        b->up_bytes = b->entries_at + sizeof(wig::World) * n;
    }
    for (uint32_t li = 0; li < WIG_BATCH_LANES; li++) {
        Lane& ln = b->lane[li];
        if (cudaMalloc(&ln.d_items, 4u * (size_t)std::max<uint64_t>(items_total, 1)) != cudaSuccess)
            return bail(WIG_E_OOM, "cudaMalloc work lists");
        if (cudaMalloc(&ln.d_count, 4u * wig::L_COUNT) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc list counts");
        cudaMemset(ln.d_count, 0, 4u * wig::L_COUNT);
        if (cudaMalloc(&ln.d_off, 4u * (size_t)wig::L_COUNT * (n + 1u)) != cudaSuccess)
            return bail(WIG_E_OOM, "cudaMalloc list offsets");
        if (cudaMalloc(&ln.d_loop, 4u) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc loop word");
        cudaMemset(ln.d_loop, 0, 4u);
        if (cudaMalloc(&ln.d_up, b->up_bytes) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc step inputs");
        cudaMemset(ln.d_up, 0, b->up_bytes);
        if (cudaMallocHost(&ln.h_up, b->up_bytes * RING) != cudaSuccess) return bail(WIG_E_OOM, "cudaMallocHost step inputs");
        for (int r = 0; r < RING; r++)
            if (cudaEventCreateWithFlags(&ln.up_ev[r], cudaEventDisableTiming) != cudaSuccess) return bail(WIG_E_CUDA, "event");
        if (cudaMalloc(&ln.d_rsub, sizeof(Report) * n) != cudaSuccess) return bail(WIG_E_OOM, "cudaMalloc lane reports");
        if (cudaMallocHost(&ln.h_rsub, sizeof(Report) * n) != cudaSuccess) return bail(WIG_E_OOM, "cudaMallocHost lane reports");
        if (cudaStreamCreateWithFlags(&ln.cap, cudaStreamNonBlocking) != cudaSuccess) return bail(WIG_E_CUDA, "stream");
        if (cudaStreamCreateWithFlags(&ln.cap2, cudaStreamNonBlocking) != cudaSuccess) return bail(WIG_E_CUDA, "stream");
        if (cudaStreamCreateWithFlags(&ln.cap3, cudaStreamNonBlocking) != cudaSuccess) return bail(WIG_E_CUDA, "stream");
        wig::Batch& Bt = ln.Bt;
        Bt.worlds = b->d_worlds;
        Bt.items = ln.d_items;
        Bt.count = ln.d_count;
        for (uint32_t l = 0; l < wig::L_COUNT; l++) Bt.base[l] = base[l];
        Bt.lbits = b->lbits;
        Bt.single = n == 1 ? 1u : 0u;
        Bt.max_cycles = 1;
        Bt.cond = 0;
        Bt.cond_check = 0;
        Bt.cond_drift = 0;
        Bt.loop = ln.d_loop;
        wig::SchedCtl& c = ln.ctl;
        c.nsub = reinterpret_cast<const uint32_t*>(ln.d_up);
        c.sub = reinterpret_cast<const uint32_t*>(ln.d_up + 8);
        c.heads = reinterpret_cast<const wig::StepHead*>(ln.d_up + 8 + ((4u * (size_t)n + 7u) & ~(size_t)7u));
        c.off = ln.d_off;
        c.items = ln.d_items;
        c.count = ln.d_count;
        c.max_worlds = n;
        c.entries = nullptr;
        c.table = nullptr;
    }
    *out = b;
    return WIG_OK;
}

void destroy_batch(wig_batch* b) {
    if (!b) return;
    cudaDeviceSynchronize();
    for (uint32_t li = 0; li < WIG_BATCH_LANES; li++) {
        Lane& ln = b->lane[li];
        drop_graphs(ln);
        if (ln.d_items) cudaFree(ln.d_items);
        if (ln.d_count) cudaFree(ln.d_count);
        if (ln.d_off) cudaFree(ln.d_off);
        if (ln.d_loop) cudaFree(ln.d_loop);
        if (ln.d_up) cudaFree(ln.d_up);
        if (ln.h_up) cudaFreeHost(ln.h_up);
        for (int r = 0; r < RING; r++)
            if (ln.up_ev[r]) cudaEventDestroy(ln.up_ev[r]);
        if (ln.d_rsub) cudaFree(ln.d_rsub);
        if (ln.h_rsub) cudaFreeHost(ln.h_rsub);
        if (ln.cap) cudaStreamDestroy(ln.cap);
        if (ln.cap2) cudaStreamDestroy(ln.cap2);
        if (ln.cap3) cudaStreamDestroy(ln.cap3);
        if (ln.d_table) cudaFree(ln.d_table);
        if (ln.d_pool) cudaFree(ln.d_pool);
    }
    for (auto& o : b->own)
        for (void* p : o)
            if (p) cudaFree(p);
    if (b->arena) cudaFree(b->arena);
    for (void* p : b->wmem)
        if (p) cudaFree(p);
    if (b->scratch) cudaFree(b->scratch);
    if (b->d_worlds) cudaFree(b->d_worlds);
    if (b->d_elems) cudaFree(b->d_elems);
    if (b->d_st) cudaFree(b->d_st);
    if (b->d_report) cudaFree(b->d_report);
    if (b->h_report) cudaFreeHost(b->h_report);
    delete b;
}

// ---------------------------------------------------------------- recording

// Per-pass timing of an eagerly launched step (the reference's per-phase
// GPU timestamps, js/timer.js:7-98): events around each launch.
struct Prof {
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
};

// Launch recording with optional per-launch events (Prof).
struct Rec {
    wig_batch* b;
    Lane& ln;
    cudaStream_t s;
    Prof* prof;
    uint32_t launches = 0;
    cudaEvent_t pending = nullptr;
    template <class Fn>
    void timed(int id, Fn fn) {
        cudaEvent_t a = nullptr, e = nullptr;
        if (prof) {
            cudaEventCreate(&a);
            cudaEventCreate(&e);
            cudaEventRecord(a, s);
        }
        fn();
        launches++;
        if (prof) {
            cudaEventRecord(e, s);
            prof->marks.push_back({id, {a, e}});
        }
    }
    void run(int pass, uint32_t level = 0, uint32_t cycle = 0) {
        timed(pass, [&] { wig::launch_pass(ln.Bt, ln.S, b->hw[0].D, pass, level, cycle, s); });
    }
    // cgStart + cgJoin as the fast forms run them (profiled as the two passes)
    void labels() {
        timed(WIG_PASS_CG_START, [&] { wig::launch_labels(ln.Bt, ln.S, s, 0); });
        timed(WIG_PASS_CG_JOIN, [&] { wig::launch_labels(ln.Bt, ln.S, s, 1); });
    }
    void norm(int which, uint32_t cycle) {
        timed(WIG_SLOT_NORM, [&] { wig::launch_norm(b->hw[0].D, which, cycle, s); });
    }
    void sched(int phase) {
        cudaEvent_t a = nullptr, e = nullptr;
        if (prof) {
            cudaEventCreate(&a);
            cudaEventCreate(&e);
            cudaEventRecord(a, s);
        }
        wig::sched_lists(ln.Bt, ln.ctl, ln.S, phase, s);
        launches += 2;
        if (prof) {
            cudaEventRecord(e, s);
            prof->marks.push_back({WIG_SLOT_SCHED, {a, e}});
        }
    }
    void report() {
        timed(WIG_SLOT_REPORT, [&] {
            k_report<<<wig::list_grid(ln.S, wig::L_ONE_ALL, 4), 32, 0, s>>>(ln.Bt, b->d_report, ln.d_rsub);
        });
    }
    // the fast form's marker hook: events around each of its launches
    static void mark(void* ctx, int slot, int phase) {
        Rec* r = static_cast<Rec*>(ctx);
        if (!r->prof) return;
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        cudaEventRecord(e, r->s);
        if (phase == 0) {
            r->pending = e;
        } else {
            r->prof->marks.push_back({slot, {r->pending, e}});
            r->pending = nullptr;
        }
    }
};

// encodeFluid's passes before the solve (js/sim.js:2486-2521), with the
// work lists written at the step's start and after compact.
// Whether the batch is one world with its free bodies bound.
bool has_bodies(const wig_batch* b) { return b->K == 1 && b->hw[0].D.motion != nullptr; }

void record_pre(Rec& R, bool viscous) {
    const bool bodies = has_bodies(R.b);
    R.sched(0);
    R.run(WIG_PASS_SYNC);
    R.run(WIG_PASS_SYNC_PARTICLES);
    R.run(WIG_PASS_SYNC_SEED);
    R.run(WIG_PASS_COMPACT);
    R.sched(1);
    R.run(WIG_PASS_RETIRE);
    R.run(WIG_PASS_CLEAR);
    R.run(WIG_PASS_GATHER);
    R.run(WIG_PASS_SEAL_JOIN);
    R.run(WIG_PASS_SEAL_ANCHOR);
    R.run(WIG_PASS_CLASSIFY);
    if (bodies) {
        R.run(WIG_PASS_BODY_START);
        R.run(WIG_PASS_BODY_LOADS);
    }
    R.run(WIG_PASS_SET_FACES);
    if (viscous)
        for (int i = 0; i < 8; i++) {
            R.run(WIG_PASS_VISCOSITY_RED);
            R.run(WIG_PASS_VISCOSITY_BLACK);
        }
    R.run(WIG_PASS_UNPRESS);
    if (bodies && viscous) {
        R.run(WIG_PASS_BODY_DRAG);
        R.run(WIG_PASS_BODY_FACES);
    }
    R.run(WIG_PASS_DIVERGENCE);
}

// encodeFluid's passes after the solve (js/sim.js:2592-2611) and the report.
void record_post(Rec& R) {
    R.run(WIG_PASS_PROJECT);
    if (has_bodies(R.b)) {
        R.run(WIG_PASS_RIGIDIFY);
        R.run(WIG_PASS_BODY_PUSH);
    }
    R.run(WIG_PASS_EXTRAPOLATE);
    R.run(WIG_PASS_EXTRAPOLATE_FURTHER);
    R.run(WIG_PASS_ADVECT);
    R.run(WIG_PASS_SORT_COUNT);
    R.run(WIG_PASS_SCAN_BLOCKS);
    R.run(WIG_PASS_SCAN_TOTALS);
    R.run(WIG_PASS_SCAN_FINISH);
    R.run(WIG_PASS_SCATTER);
    R.run(WIG_PASS_RASTER_CLAIMS);
    R.run(WIG_PASS_RASTER);
    R.run(WIG_PASS_UNPAINT);
    R.report();
}

// A single world's bookkeeping-only step (js/sim.js:2480-2485).
uint32_t record_book(Rec& R) {
    R.sched(0);
    R.run(WIG_PASS_SYNC_MARKS);
    R.run(WIG_PASS_COMPACT);
    R.sched(1);
    R.run(WIG_PASS_RETIRE);
    R.report();
    return R.launches;
}

// Records the plain form's step of world 0 (one kernel per reference pass,
// every iteration encoded) on stream s; returns the kernels launched.
uint32_t record_step(wig_batch* b, Lane& ln, uint32_t max_cycles, uint32_t flags, bool shifted, cudaStream_t s, Prof* prof) {
    Rec R{b, ln, s, prof};
    const bool tol = (flags & WIG_STEP_TOLERANCE) != 0u;
    if (flags & WIG_STEP_BOOKKEEPING_ONLY) return record_book(R);
    record_pre(R, (flags & WIG_STEP_VISCOUS) != 0u);
    const uint32_t deepest = b->L[0].levels;
    R.run(WIG_PASS_CG_START);
    R.run(WIG_PASS_CG_JOIN);
    R.run(WIG_PASS_CG_ANCHOR);
    const bool bodies = has_bodies(b);
    if (bodies) R.run(WIG_PASS_CG_BODY_X);
    R.run(WIG_PASS_CG_RESIDUAL);
    if (tol) R.norm(0, 0);
    R.run(WIG_PASS_CG_PREPARE);
    bool sh = shifted;
    for (uint32_t cycle = 0; cycle < max_cycles; cycle++) {
        R.run(WIG_PASS_RELAX_RIMS, 0, cycle);
        R.run(sh ? WIG_PASS_RELAX_SHIFTED : WIG_PASS_RELAX, 0, cycle);
        sh = !sh;
        for (uint32_t l = 1; l <= deepest; l++) {
            R.run(WIG_PASS_RESTRICT, l, cycle);
            if (l < deepest) {
                R.run(WIG_PASS_SMOOTH_RED, l, cycle);
                R.run(WIG_PASS_SMOOTH_BLACK, l, cycle);
            }
        }
        R.run(WIG_PASS_SOLVE, deepest, cycle);
        for (uint32_t l = deepest - 1; l >= 1; l--) {
            R.run(WIG_PASS_PROLONG, l, cycle);
            R.run(WIG_PASS_SMOOTH_RED, l, cycle);
            R.run(WIG_PASS_SMOOTH_BLACK, l, cycle);
        }
        R.run(WIG_PASS_PROLONG_FINE, 0, cycle);
        R.run(WIG_PASS_RELAX_RIMS, 0, cycle);
        R.run(sh ? WIG_PASS_RELAX_SHIFTED : WIG_PASS_RELAX, 0, cycle);
        sh = !sh;
        R.run(WIG_PASS_CG_RHO, 0, cycle);
        R.run(WIG_PASS_CG_BETA, 0, cycle);
        R.run(WIG_PASS_CG_DIRECTION, 0, cycle);
        if (bodies) R.run(WIG_PASS_CG_BODY_P, 0, cycle);
        R.run(WIG_PASS_CG_APPLY, 0, cycle);
        R.run(WIG_PASS_CG_ALPHA, 0, cycle);
        R.run(WIG_PASS_CG_UPDATE, 0, cycle);
        if (tol) R.norm(1, cycle);
    }
    R.run(WIG_PASS_CG_FINISH);
    if (bodies) R.run(WIG_PASS_CG_BODY_F);
    record_post(R);
    return R.launches;
}

// Records the fast form's step of the lane's worlds.  With `capture`, s is
// capturing into a graph and the iterations become a WHILE node whose body
// is captured on the lane's second stream; else the iterations are launched
// from the host, each decided by reading back the device's verdict (the
// profiler's path).  *outside gets the kernels outside the loop (all of
// them when not capturing), *body those of one iteration of the loop.  The
// persistent form (one world) runs the iterations in one cooperative kernel.
int record_step_fast(wig_batch* b, Lane& ln, uint32_t max_cycles, uint32_t flags, bool shifted, cudaStream_t s,
                     Prof* prof, bool capture, uint32_t* outside, uint32_t* body) {
    Rec R{b, ln, s, prof};
    if ((flags & WIG_STEP_BOOKKEEPING_ONLY) && b->K == 1) {
        *outside = record_book(R);
        *body = 0;
        return WIG_OK;
    }
    record_pre(R, (flags & WIG_STEP_VISCOUS) != 0u);
    R.labels();
    R.run(WIG_PASS_CG_ANCHOR);
    wig::Marker mk{&Rec::mark, &R};
    ln.Bt.max_cycles = max_cycles;
    ln.Bt.cond = 0;
    ln.Bt.cond_check = 0;
    ln.Bt.cond_drift = 0;
    ln.Bt.mixed = (flags & WIG_STEP_MIXED) ? 1u : 0u;
    const wig::World* one = b->K == 1 ? &b->hw[0] : nullptr;
    if (b->pooled) {
        wig::fast_zero_idle(ln.Bt, ln.S, s);
        R.launches++;
    }
    wig::fast_setup(ln.Bt, ln.S, one, s, prof ? &mk : nullptr);
    R.launches++;
    if (flags & WIG_STEP_PERSISTENT) {
        wig::Fast F0;
        static_cast<wig::FastW&>(F0) = b->hw[0].S;
        F0.D = b->hw[0].D;
        F0.max_cycles = max_cycles;
        F0.solve_grid = b->solve_grid;
        if (F0.solve_grid == 0u) return fail(WIG_E_STATE, "no grid for the persistent solve");
        CUDA_TRY(wig::fast_solve(F0, shifted, s, prof ? &mk : nullptr));
        R.launches++;
        *body = 0;
    } else if (capture) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        CUDA_TRY(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
        cudaGraphConditionalHandle handle;
        CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        CUDA_TRY(cudaGraphAddNode(&cnode, g, deps, nd, &cp));
        CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies));
        cudaGraph_t bodyGraph = cp.conditional.phGraph_out[0];
        CUDA_TRY(cudaStreamBeginCaptureToGraph(ln.cap2, bodyGraph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        wig::Batch Bc = ln.Bt;
        Bc.cond = (unsigned long long)handle;
        wig::NestCapture nest{ln.cap3, cudaSuccess};
        *body = wig::fast_cycle(Bc, ln.S, one, ln.cap2, nullptr, &nest);
        cudaGraph_t captured = nullptr;
        CUDA_TRY(cudaStreamEndCapture(ln.cap2, &captured));
        CUDA_TRY(nest.err);
    } else {
        uint32_t* cont = reinterpret_cast<uint32_t*>(ln.h_rsub);  // a word of pinned scratch
        for (uint32_t c = 0; c < max_cycles; c++) {
            R.launches += wig::fast_cycle(ln.Bt, ln.S, one, s, prof ? &mk : nullptr);
            CUDA_TRY(cudaMemcpyAsync(cont, ln.d_loop, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaStreamSynchronize(s));
            if (!*cont) break;
        }
        *body = 0;
    }
    wig::fast_finish(ln.Bt, ln.S, one, (flags & WIG_STEP_PERSISTENT) == 0u, s, prof ? &mk : nullptr);
    R.launches++;
    record_post(R);
    *outside = R.launches;
    return WIG_OK;
}

// ---------------------------------------------------------------- stepping

struct StepArgs {
    uint32_t lane;
    const uint32_t* worlds;
    uint32_t count;
    const wig_params* P;
    const uint32_t* world_flags;  // null: `flags`' per-world bits for all
    uint32_t max_cycles;
    uint32_t flags;
    double tol;
    cudaStream_t s;
};

constexpr uint32_t WORLD_BITS = WIG_STEP_BOOKKEEPING_ONLY | WIG_STEP_VISCOUS | WIG_STEP_SHIFTED_SET | WIG_STEP_SHIFTED_FIRST;

int check_step(wig_batch* b, const StepArgs& a) {
    if (!b || !a.worlds || !a.P) return fail(WIG_E_ARG, "null argument");
    if (a.lane >= WIG_BATCH_LANES) return fail(WIG_E_ARG, "lane out of range");
    if (a.count == 0 || a.count > b->K) return fail(WIG_E_ARG, "world count out of range");
    if (a.max_cycles == 0 || a.max_cycles > 64) return fail(WIG_E_ARG, "max_cycles out of range (1..64)");
    if ((a.flags & WIG_STEP_TOLERANCE) && !(a.tol > 0.0)) return fail(WIG_E_ARG, "tolerance must be positive");
    if ((a.flags & (WIG_STEP_PLAIN | WIG_STEP_PERSISTENT)) && b->K != 1)
        return fail(WIG_E_ARG, "the plain and persistent forms step one world");
    if ((a.flags & WIG_STEP_MIXED) &&
        ((a.flags & (WIG_STEP_PLAIN | WIG_STEP_PERSISTENT)) ||
         (a.flags & (WIG_STEP_TOLERANCE | WIG_STEP_F64_DOTS)) != (WIG_STEP_TOLERANCE | WIG_STEP_F64_DOTS)))
        return fail(WIG_E_ARG, "the mixed form is a fast form with WIG_STEP_TOLERANCE and WIG_STEP_F64_DOTS");
    std::vector<char> seen(b->K, 0);
    for (uint32_t i = 0; i < a.count; i++) {
        const uint32_t k = a.worlds[i];
        if (k >= b->K) return fail(WIG_E_ARG, "world index out of range");
        if (seen[k]) return fail(WIG_E_ARG, "a world listed twice");
        seen[k] = 1;
        if (!b->bound[k]) return fail(WIG_E_STATE, "buffers not bound");
    }
    return WIG_OK;
}

// Writes the step's inputs into the lane's next pinned slot and copies them
// to the device; returns the batch-wide viscous bit and (one world) the
// tiling parity of its step.
int push_inputs(wig_batch* b, Lane& ln, const StepArgs& a, bool* viscous, bool* shifted0) {
    const int r = ln.up_at;
    ln.up_at = (ln.up_at + 1) % RING;
    CUDA_TRY(cudaEventSynchronize(ln.up_ev[r]));
    char* slot = ln.h_up + b->up_bytes * r;
    const size_t sub_bytes = (4u * (size_t)b->K + 7u) & ~(size_t)7u;
    uint32_t* hdr = reinterpret_cast<uint32_t*>(slot);
    uint32_t* sub = reinterpret_cast<uint32_t*>(slot + 8);
    wig::StepHead* heads = reinterpret_cast<wig::StepHead*>(slot + 8 + sub_bytes);
    hdr[0] = a.count;
    hdr[1] = 0u;
    *viscous = false;
    *shifted0 = false;
    for (uint32_t i = 0; i < a.count; i++) {
        const uint32_t k = a.worlds[i];
        const uint32_t wf = (a.world_flags ? a.world_flags[i] : a.flags) & WORLD_BITS;
        sub[i] = k;
        wig::StepHead& h = heads[i];
        std::memset(&h, 0, sizeof(h));
        h.P = a.P[i];
        h.P.size[0] = b->L[k].width;
        h.P.size[1] = b->L[k].height;
        h.tol_mode = (a.flags & WIG_STEP_TOLERANCE) ? 1u : 0u;
        h.f64 = (a.flags & WIG_STEP_F64_DOTS) ? 1u : 0u;
        h.book = (wf & WIG_STEP_BOOKKEEPING_ONLY) ? 1u : 0u;
        h.viscous = (wf & WIG_STEP_VISCOUS) ? 1u : 0u;
        bool sh;
        if (wf & WIG_STEP_SHIFTED_SET) {
            sh = (wf & WIG_STEP_SHIFTED_FIRST) != 0u;
        } else {
            if (!h.book) b->shifted_first[k] = !b->shifted_first[k];
            sh = b->shifted_first[k] != 0;
        }
        h.shift_first = sh ? 1u : 0u;
        h.tol = a.tol;
        *viscous = *viscous || h.viscous;
        if (i == 0) *shifted0 = sh;
    }
    const size_t bytes = 8u + sub_bytes + sizeof(wig::StepHead) * a.count;
    if (b->pooled) {
        // each stepping world's per-step memory from the lane's pool
        if (!ln.d_pool) return fail(WIG_E_STATE, "the lane has no pool");
        wig::World* ent = reinterpret_cast<wig::World*>(slot + b->entries_at);
        uint64_t at = 0;
        for (uint32_t i = 0; i < a.count; i++) {
            const uint32_t k = a.worlds[i];
            const uint64_t need = transient_bytes(b->L[k], b->hw[k].D);
            if (at + need > ln.pool_bytes) return fail(WIG_E_OOM, "the step's worlds do not fit the lane's pool");
            wig::World e = b->hw[k];
            char* q = ln.d_pool + at;
            e.D.parts = reinterpret_cast<uint32_t*>(q);
            q += align256(buffer_bytes(b->L[k], 2));
            e.D.cg = reinterpret_cast<float*>(q);
            q += align256(buffer_bytes(b->L[k], 6));
            scratch_take(e, q, b->S.coarse_cells);
            ent[i] = e;
            at += need;
        }
        CUDA_TRY(cudaMemcpyAsync(ln.d_up + b->entries_at, ent, sizeof(wig::World) * a.count, cudaMemcpyHostToDevice, a.s));
    }
    // the heads sit after the full sub array, so copy the slot's prefix
    // through the last head written
    CUDA_TRY(cudaMemcpyAsync(ln.d_up, slot, bytes, cudaMemcpyHostToDevice, a.s));
    CUDA_TRY(cudaEventRecord(ln.up_ev[r], a.s));
    return WIG_OK;
}

// Level 0 of the listed worlds whose buffers the host has written since
// their last step, zeroed (the fast form's invariant).
void zero_dirty(wig_batch* b, const StepArgs& a) {
    if (b->pooled) return;  // the step zeroes its lent scratch itself
    for (uint32_t i = 0; i < a.count; i++) {
        const uint32_t k = a.worlds[i];
        if (!b->dirty[k]) continue;
        wig::fast_zero_level0(b->hw[k].S, b->hw[k].D.C, a.s);
        b->dirty[k] = 0;
    }
}

// The shape a step records with: every list's grid sized for the step's
// worlds rather than the whole batch's, by their blocks rounded up to a
// power of two (`bucket`, part of the graph's key) against all the
// batch's blocks, so a small step of a large batch launches no idle CTAs
// by the thousand.  A grid's size changes no result.
wig::BatchShape step_shape(const wig_batch* b, const StepArgs& a, uint32_t* bucket) {
    wig::BatchShape S = b->S;
    uint64_t blocks = 0;
    for (uint32_t i = 0; i < a.count; i++) blocks += b->hw[a.worlds[i]].D.B;
    uint32_t e = 0;
    while (e < 48u && (1ull << e) < blocks) e++;
    *bucket = e;
    const double f = (double)(1ull << e) / (double)std::max<uint64_t>(b->blocks_all, 1);
    if (f < 1.0) {
        for (uint32_t l = 0; l < wig::L_COUNT; l++)
            S.max_items[l] = (uint32_t)std::max(1.0, std::ceil((double)S.max_items[l] * f));
        S.worlds = (uint32_t)std::max(1.0, std::ceil((double)S.worlds * f));
    }
    return S;
}

int batch_step(wig_batch* b, const StepArgs& a) {
    int rc = check_step(b, a);
    if (rc) return rc;
    Lane& ln = b->lane[a.lane];
    bool viscous = false, sh = false;
    rc = push_inputs(b, ln, a, &viscous, &sh);
    if (rc) return rc;
    const bool plain = (a.flags & WIG_STEP_PLAIN) != 0u;
    if (!plain) zero_dirty(b, a);
    const bool book1 = b->K == 1 && ((a.world_flags ? a.world_flags[0] : a.flags) & WIG_STEP_BOOKKEEPING_ONLY) != 0u;
    uint32_t shape = a.flags & (WIG_STEP_TOLERANCE | WIG_STEP_F64_DOTS | WIG_STEP_PLAIN | WIG_STEP_PERSISTENT | WIG_STEP_MIXED);
    if (viscous) shape |= WIG_STEP_VISCOUS;
    if (book1) shape |= WIG_STEP_BOOKKEEPING_ONLY;
    const bool parity_keyed = plain || (a.flags & WIG_STEP_PERSISTENT);
    uint32_t bucket = 0;
    ln.S = step_shape(b, a, &bucket);
    const uint64_t key = ((uint64_t)a.max_cycles << 32) | ((uint64_t)bucket << 24) | ((uint64_t)shape << 1) |
                         ((parity_keyed && sh) ? 1u : 0u);
    auto it = ln.graphs.find(key);
    if (it == ln.graphs.end()) {
        Graph G;
        CUDA_TRY(cudaStreamBeginCapture(ln.cap, cudaStreamCaptureModeThreadLocal));
        uint32_t n = 0, nb = 0;
        if (plain) {
            n = record_step(b, ln, a.max_cycles, shape, sh, ln.cap, nullptr);
        } else {
            int rc2 = record_step_fast(b, ln, a.max_cycles, shape, sh, ln.cap, nullptr, true, &n, &nb);
            if (rc2) {
                std::string m = g_last_error;
                cudaGraph_t junk = nullptr;
                cudaStreamEndCapture(ln.cap, &junk);
                if (junk) cudaGraphDestroy(junk);
                return fail(rc2, m);
            }
        }
        cudaError_t e = cudaStreamEndCapture(ln.cap, &G.g);
        if (e != cudaSuccess) return fail(WIG_E_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&G.ge, G.g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(G.g);
            return fail(WIG_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        G.outside = n;
        G.body = nb;
        it = ln.graphs.emplace(key, G).first;
    }
    ln.last_launches = it->second.outside;
    ln.last_body = it->second.body;
    CUDA_TRY(cudaGraphLaunch(it->second.ge, a.s));
    if (a.flags & WIG_STEP_SYNC_STATS)
        CUDA_TRY(cudaMemcpyAsync(ln.h_rsub, ln.d_rsub, sizeof(Report) * a.count, cudaMemcpyDeviceToHost, a.s));
    ln.last_stream = a.s;
    for (uint32_t i = 0; i < a.count; i++) {
        b->stepped_on[a.worlds[i]] = a.s;
        b->stepped_lane[a.worlds[i]] = (int)a.lane;
    }
    return WIG_OK;
}

int batch_step_profile(wig_batch* b, const StepArgs& a, float* ms_out, uint32_t* calls_out) {
    if (!ms_out || !calls_out) return fail(WIG_E_ARG, "null argument");
    int rc = check_step(b, a);
    if (rc) return rc;
    Lane& ln = b->lane[a.lane];
    bool viscous = false, sh = false;
    rc = push_inputs(b, ln, a, &viscous, &sh);
    if (rc) return rc;
    const bool plain = (a.flags & WIG_STEP_PLAIN) != 0u;
    const bool book1 = b->K == 1 && ((a.world_flags ? a.world_flags[0] : a.flags) & WIG_STEP_BOOKKEEPING_ONLY) != 0u;
    uint32_t shape = a.flags & (WIG_STEP_TOLERANCE | WIG_STEP_F64_DOTS | WIG_STEP_PLAIN | WIG_STEP_PERSISTENT | WIG_STEP_MIXED);
    if (viscous) shape |= WIG_STEP_VISCOUS;
    if (book1) shape |= WIG_STEP_BOOKKEEPING_ONLY;
    Prof prof;
    ln.last_body = 0;
    uint32_t bucket = 0;
    ln.S = step_shape(b, a, &bucket);
    if (plain) {
        ln.last_launches = record_step(b, ln, a.max_cycles, shape, sh, a.s, &prof);
    } else {
        zero_dirty(b, a);
        uint32_t n = 0, nb = 0;
        rc = record_step_fast(b, ln, a.max_cycles, shape, sh, a.s, &prof, false, &n, &nb);
        if (rc) return rc;
        ln.last_launches = n;
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(a.s));
    for (int k = 0; k < WIG_PROFILE_SLOTS; k++) { ms_out[k] = 0.0f; calls_out[k] = 0u; }
    for (auto& m : prof.marks) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, m.second.first, m.second.second);
        ms_out[m.first] += ms;
        calls_out[m.first] += 1u;
        cudaEventDestroy(m.second.first);
        cudaEventDestroy(m.second.second);
    }
    ln.last_stream = a.s;
    for (uint32_t i = 0; i < a.count; i++) {
        b->stepped_on[a.worlds[i]] = a.s;
        b->stepped_lane[a.worlds[i]] = (int)a.lane;
    }
    return WIG_OK;
}

int severity(int rc) {
    switch (rc) {
    case WIG_OK: return 0;
    case WIG_E_NOT_CONVERGED: return 1;
    case WIG_E_CAPACITY: return 2;
    default: return 3;
    }
}

int batch_read_stats(wig_batch* b, const uint32_t* worlds, uint32_t count, wig_fluid_stats* out) {
    if (!b || !worlds || !out) return fail(WIG_E_ARG, "null argument");
    std::vector<cudaStream_t> waited;
    for (uint32_t i = 0; i < count; i++) {
        if (worlds[i] >= b->K) return fail(WIG_E_ARG, "world index out of range");
        cudaStream_t s = b->stepped_on[worlds[i]];
        bool done = false;
        for (cudaStream_t w : waited) done = done || w == s;
        if (!done) {
            CUDA_TRY(cudaStreamSynchronize(s));
            waited.push_back(s);
        }
    }
    int rc = WIG_OK;
    // one copy of every world's report when more than a few are asked for
    const bool all = count > 4;
    if (all) CUDA_TRY(cudaMemcpy(b->h_report, b->d_report, sizeof(Report) * b->K, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < count; i++) {
        const uint32_t k = worlds[i];
        if (!all) CUDA_TRY(cudaMemcpy(&b->h_report[k], &b->d_report[k], sizeof(Report), cudaMemcpyDeviceToHost));
        const Report& r = b->h_report[k];
        wig_fluid_stats& o = out[i];
        std::memset(&o, 0, sizeof(o));
        for (uint32_t c = 0; c < WIG_FLUID_STATS; c++) o.count[c] = r.count[c];
        o.particles = r.particles;
        o.cycles = r.count[WIG_COUNT_CYCLES];
        const int li = b->stepped_lane[k];
        if (li >= 0) o.launches = b->lane[li].last_launches + b->lane[li].last_body * r.count[WIG_COUNT_CYCLES];
        o.rel_residual = r.rel;
        o.b_norm = r.bnorm2 > 0.0 ? __builtin_sqrt(r.bnorm2) : 0.0;
        o.true_residual = r.rel_true;
        // the most severe of the worlds' conditions is returned, every
        // world's report filled in all the same: a device loop that gave up,
        // then particles past the capacity, then a solve short of its
        // tolerance
        if (r.err & wig::ERR_BARRIER) {
            if (severity(rc) < severity(WIG_E_STATE))
                rc = fail(WIG_E_STATE, "the persistent solve's grid barrier waited past its limit");
        } else if (r.err) {
            if (severity(rc) < severity(WIG_E_STATE))
                rc = fail(WIG_E_STATE, "a device loop hit its iteration limit (union-find)");
        } else if (r.tried > b->L[k].capacity) {
            if (severity(rc) < severity(WIG_E_CAPACITY))
                rc = fail(WIG_E_CAPACITY, "world " + std::to_string(k) + ": " + std::to_string(r.tried) +
                                              " particles for room for " + std::to_string(b->L[k].capacity) +
                                              "; those past the room were lost");
        } else if (r.short_of_tol) {
            if (severity(rc) < severity(WIG_E_NOT_CONVERGED))
                rc = fail(WIG_E_NOT_CONVERGED, "world " + std::to_string(k) + ": the solve left a relative residual of " +
                                                   std::to_string(r.rel) + " after " +
                                                   std::to_string(r.count[WIG_COUNT_CYCLES]) + " iterations");
        }
    }
    return rc;
}

int copy_world(wig_batch* b, uint32_t k, int which, void* host, uint64_t offset, uint64_t bytes, void* stream, bool up) {
    if (!b || !host) return fail(WIG_E_ARG, "null argument");
    if (k >= b->K) return fail(WIG_E_ARG, "world index out of range");
    if (!b->bound[k]) return fail(WIG_E_STATE, "buffers not bound");
    uint64_t size = buffer_bytes(b->L[k], which);
    if (!size || offset > size || bytes > size - offset)
        return fail(WIG_E_ARG, up ? "upload out of the buffer's range" : "download out of the buffer's range");
    if (b->pooled && borrowed(which)) return fail(WIG_E_STATE, "`parts` and `cg` are per-step memory in a pooled batch");
    if (b->pooled && which == 4) {
        // a pooled world's field ends before its coarse levels
        const uint64_t kept = persistent_buffer_bytes(b->L[k], 4);
        if (offset > kept) return fail(WIG_E_ARG, "field past a pooled world's kept part");
        if (bytes > kept - offset) bytes = kept - offset;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char* dev = (char*)*buffer_slot(b->hw[k].D, which) + offset;
    if (up) CUDA_TRY(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
    else CUDA_TRY(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (up) b->dirty[k] = 1;
    return WIG_OK;
}

}  // namespace

extern "C" {

uint32_t wig_fluid_abi_version(void) { return WIG_ABI_VERSION; }

int wig_fluid_set_wait_limits(uint32_t loop_limit, uint32_t spin_limit) {
    const uint32_t lo = loop_limit ? loop_limit : wig::LOOP_LIMIT;
    const uint32_t sp = spin_limit ? spin_limit : wig::BARRIER_SPIN_LIMIT;
    if (lo > wig::LOOP_LIMIT || sp > wig::BARRIER_SPIN_LIMIT)
        return fail(WIG_E_ARG, "wait limits may only be lowered");
    CUDA_TRY(cudaMemcpyToSymbol(wig::g_loop_limit, &lo, sizeof(lo)));
    CUDA_TRY(cudaMemcpyToSymbol(wig::g_spin_limit, &sp, sizeof(sp)));
    return WIG_OK;
}

const char* wig_fluid_last_error(void) { return g_last_error.c_str(); }

int wig_fluid_layout(const wig_world_desc* d, wig_world_layout* out) { return layout_of(d, out); }

int wig_fluid_create(const wig_world_desc* d, const wig_elem* elems, uint32_t n_elems, wig_fluid** out) {
    if (!out) return fail(WIG_E_ARG, "null output handle");
    *out = nullptr;
    if (!d) return fail(WIG_E_ARG, "null descriptor");
    wig_fluid* h = new (std::nothrow) wig_fluid();
    if (!h) return fail(WIG_E_OOM, "host allocation failed");
    int rc = make_batch(d, 1, elems, n_elems, Alloc::Single, &h->b);
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return WIG_OK;
}

int wig_fluid_bind(wig_fluid* h, const wig_fluid_buffers* bufs) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null handle");
    wig_batch* b = h->b;
    for (auto& ln : b->lane) drop_graphs(ln);
    void* given[7] = {nullptr};
    if (bufs) {
        given[0] = bufs->cells; given[1] = bufs->sorted; given[2] = bufs->parts; given[3] = bufs->counters;
        given[4] = bufs->field; given[5] = bufs->blocks; given[6] = bufs->cg;
    }
    wig::Dev& D = b->hw[0].D;
    for (int k = 0; k < 7; k++) {
        void** slot = buffer_slot(D, k);
        if (given[k]) {
            if (((uintptr_t)given[k] & 15u) != 0u) return fail(WIG_E_ARG, "buffer not 16-byte aligned");
            if (b->own[0][k]) { cudaFree(b->own[0][k]); b->own[0][k] = nullptr; }
            *slot = given[k];
        } else if (!b->own[0][k]) {
            uint64_t bytes = buffer_bytes(b->L[0], k);
            void* p = nullptr;
            if (cudaMalloc(&p, bytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(WIG_E_OOM, "cudaMalloc of a world buffer failed");
            }
            CUDA_TRY(cudaMemset(p, 0, bytes));
            b->own[0][k] = p;
            *slot = p;
        }
    }
    int rc = upload_world_entry(b, 0);
    if (rc) return rc;
    b->bound[0] = 1;
    b->dirty[0] = 1;
    return WIG_OK;
}

int wig_fluid_bind_bodies(wig_fluid* h, void* motion, void* pushes, void* stamps) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null handle");
    if ((motion == nullptr) != (pushes == nullptr)) return fail(WIG_E_ARG, "bind both body buffers or neither");
    if (((uintptr_t)motion & 15u) != 0u || ((uintptr_t)pushes & 15u) != 0u || ((uintptr_t)stamps & 15u) != 0u)
        return fail(WIG_E_ARG, "body buffer not 16-byte aligned");
    wig_batch* b = h->b;
    for (auto& ln : b->lane) drop_graphs(ln);
    b->hw[0].D.motion = static_cast<uint32_t*>(motion);
    b->hw[0].D.pushes = static_cast<uint32_t*>(pushes);
    b->hw[0].D.stamps = motion ? static_cast<uint32_t*>(stamps) : nullptr;
    return upload_world_entry(b, 0);
}

// A world with its free bodies bound steps in the plain form (the coupled
// operator is the reference's pass sequence, fluid.wgsl:2819-2845).
uint32_t step_flags_of(const wig_fluid* h, uint32_t flags) {
    if (!has_bodies(h->b)) return flags;
    return (flags | WIG_STEP_PLAIN) & ~(WIG_STEP_PERSISTENT | WIG_STEP_MIXED);
}

int wig_fluid_buffers_of(wig_fluid* h, wig_fluid_buffers* out) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null argument");
    return wig_batch_buffers_of(h->b, 0, out);
}

int wig_fluid_upload(wig_fluid* h, int which, const void* host, uint64_t offset, uint64_t bytes, void* stream) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null argument");
    return copy_world(h->b, 0, which, const_cast<void*>(host), offset, bytes, stream, true);
}

int wig_fluid_download(wig_fluid* h, int which, void* host, uint64_t offset, uint64_t bytes, void* stream) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null argument");
    return copy_world(h->b, 0, which, host, offset, bytes, stream, false);
}

int wig_fluid_dispatch(wig_fluid* h, const wig_params* P, int pass, uint32_t level, uint32_t cycle, void* stream) {
    if (!h || !h->b || !P) return fail(WIG_E_ARG, "null argument");
    wig_batch* b = h->b;
    if (!b->bound[0]) return fail(WIG_E_STATE, "buffers not bound");
    if (pass < 0 || pass >= WIG_PASS_COUNT) return fail(WIG_E_ARG, "unknown pass");
    if (level > b->L[0].levels) return fail(WIG_E_ARG, "level past the coarsest");
    cudaStream_t s = (cudaStream_t)stream;
    Lane& ln = b->lane[0];
    // the pass runs as asked: Params written, world 0 the whole subset, not
    // bookkeeping-only, with its viscosity sweeps
    wig_params p = *P;
    p.size[0] = b->L[0].width;
    p.size[1] = b->L[0].height;
    const int r = ln.up_at;
    ln.up_at = (ln.up_at + 1) % RING;
    CUDA_TRY(cudaEventSynchronize(ln.up_ev[r]));
    char* slot = ln.h_up + b->up_bytes * r;
    uint32_t* hdr = reinterpret_cast<uint32_t*>(slot);
    hdr[0] = 1u;
    hdr[1] = 0u;
    hdr[2] = 0u;
    std::memcpy(slot + 16, &p, sizeof(p));
    const uint32_t flags2[2] = {0u, 1u};  // book, viscous
    std::memcpy(slot + 16 + sizeof(p), flags2, sizeof(flags2));
    CUDA_TRY(cudaMemcpyAsync(ln.d_up, slot, 12, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(&b->d_st[0].P, slot + 16, sizeof(p), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(&b->d_st[0].book, slot + 16 + sizeof(p), sizeof(flags2), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaEventRecord(ln.up_ev[r], s));
    wig::SchedCtl c = ln.ctl;
    c.heads = nullptr;
    wig::sched_lists(ln.Bt, c, b->S, 0, s);
    wig::sched_lists(ln.Bt, c, b->S, 1, s);
    int rc = wig::launch_pass(ln.Bt, b->S, b->hw[0].D, pass, level, cycle, s);
    if (rc) return fail(rc, "launch");
    CUDA_TRY(cudaGetLastError());
    ln.last_stream = s;
    b->stepped_on[0] = s;
    return WIG_OK;
}

int wig_fluid_step(wig_fluid* h, const wig_params* P, uint32_t max_cycles, uint32_t flags, double tolerance, void* stream) {
    if (!h || !h->b || !P) return fail(WIG_E_ARG, "null argument");
    const uint32_t w0 = 0;
    StepArgs a{0, &w0, 1, P, nullptr, max_cycles, step_flags_of(h, flags), tolerance, (cudaStream_t)stream};
    return batch_step(h->b, a);
}

int wig_fluid_step_profile(wig_fluid* h, const wig_params* P, uint32_t max_cycles, uint32_t flags, double tolerance,
                           void* stream, float* ms_out, uint32_t* calls_out) {
    if (!h || !h->b || !P) return fail(WIG_E_ARG, "null argument");
    const uint32_t w0 = 0;
    StepArgs a{0, &w0, 1, P, nullptr, max_cycles, step_flags_of(h, flags), tolerance, (cudaStream_t)stream};
    return batch_step_profile(h->b, a, ms_out, calls_out);
}

int wig_fluid_set_launch(wig_fluid* h, uint32_t knob, uint32_t value) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null handle");
    return wig_batch_set_launch(h->b, knob, value);
}

int wig_fluid_get_launch(const wig_fluid* h, uint32_t knob, uint32_t* value) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null handle");
    return wig_batch_get_launch(h->b, knob, value);
}

int wig_fluid_read_stats(wig_fluid* h, wig_fluid_stats* out) {
    if (!h || !h->b) return fail(WIG_E_ARG, "null argument");
    const uint32_t w0 = 0;
    return batch_read_stats(h->b, &w0, 1, out);
}

void wig_fluid_destroy(wig_fluid* h) {
    if (!h) return;
    destroy_batch(h->b);
    delete h;
}

// ---------------------------------------------------------------- batches

int wig_batch_world_bytes(const wig_world_desc* d, uint64_t* out) {
    if (!out) return fail(WIG_E_ARG, "null argument");
    wig_world_layout L;
    int rc = layout_of(d, &L);
    if (rc) return rc;
    wig::Dev D{};
    dev_shape(D, L);
    *out = world_buffers_bytes(L) + scratch_bytes(D) + sizeof(wig::StepState) + sizeof(wig::World) + 3u * sizeof(Report);
    return WIG_OK;
}

int wig_batch_create(const wig_world_desc* descs, uint32_t n, const wig_elem* elems, uint32_t n_elems, wig_batch** out) {
    return make_batch(descs, n, elems, n_elems, Alloc::Packed, out);
}

uint32_t wig_batch_worlds(const wig_batch* b) { return b ? b->K : 0u; }

int wig_batch_layout(const wig_batch* b, uint32_t world, wig_world_layout* out) {
    if (!b || !out) return fail(WIG_E_ARG, "null argument");
    if (world >= b->K) return fail(WIG_E_ARG, "world index out of range");
    *out = b->L[world];
    return WIG_OK;
}

int wig_batch_buffers_of(wig_batch* b, uint32_t world, wig_fluid_buffers* out) {
    if (!b || !out) return fail(WIG_E_ARG, "null argument");
    if (world >= b->K) return fail(WIG_E_ARG, "world index out of range");
    if (!b->bound[world]) return fail(WIG_E_STATE, "buffers not bound");
    const wig::Dev& D = b->hw[world].D;
    out->cells = D.cells; out->sorted = D.sorted; out->parts = D.parts; out->counters = D.counters;
    out->field = D.field; out->blocks = D.blocks; out->cg = D.cg;
    return WIG_OK;
}

int wig_batch_upload(wig_batch* b, uint32_t world, int which, const void* host, uint64_t offset, uint64_t bytes,
                     void* stream) {
    return copy_world(b, world, which, const_cast<void*>(host), offset, bytes, stream, true);
}

int wig_batch_download(wig_batch* b, uint32_t world, int which, void* host, uint64_t offset, uint64_t bytes,
                       void* stream) {
    return copy_world(b, world, which, host, offset, bytes, stream, false);
}

int wig_batch_step(wig_batch* b, uint32_t lane, const uint32_t* worlds, uint32_t count, const wig_params* P,
                   const uint32_t* world_flags, uint32_t max_cycles, uint32_t flags, double tolerance, void* stream) {
    if (flags & (WIG_STEP_PLAIN | WIG_STEP_PERSISTENT)) return fail(WIG_E_ARG, "a batch steps in the fast form");
    StepArgs a{lane, worlds, count, P, world_flags, max_cycles, flags & ~WORLD_BITS, tolerance, (cudaStream_t)stream};
    if (!world_flags) a.world_flags = nullptr;
    return batch_step(b, a);
}

int wig_batch_read_stats(wig_batch* b, const uint32_t* worlds, uint32_t count, wig_fluid_stats* out) {
    return batch_read_stats(b, worlds, count, out);
}

int wig_batch_step_profile(wig_batch* b, uint32_t lane, const uint32_t* worlds, uint32_t count, const wig_params* P,
                           const uint32_t* world_flags, uint32_t max_cycles, uint32_t flags, double tolerance,
                           void* stream, float* ms_out, uint32_t* calls_out) {
    if (flags & (WIG_STEP_PLAIN | WIG_STEP_PERSISTENT)) return fail(WIG_E_ARG, "a batch steps in the fast form");
    StepArgs a{lane, worlds, count, P, world_flags, max_cycles, flags & ~WORLD_BITS, tolerance, (cudaStream_t)stream};
    return batch_step_profile(b, a, ms_out, calls_out);
}

void wig_batch_destroy(wig_batch* b) { destroy_batch(b); }

int wig_batch_create_deferred(const wig_world_desc* descs, uint32_t n, const wig_elem* elems, uint32_t n_elems,
                              wig_batch** out) {
    return make_batch(descs, n, elems, n_elems, Alloc::Deferred, out);
}

int wig_batch_admit(wig_batch* b, uint32_t world, void* stream) {
    if (!b) return fail(WIG_E_ARG, "null batch");
    if (world >= b->K) return fail(WIG_E_ARG, "world index out of range");
    if (b->wmem.empty()) return fail(WIG_E_STATE, "not a deferred batch");
    if (b->wmem[world]) return fail(WIG_E_STATE, "world already admitted");
    cudaStream_t s = (cudaStream_t)stream;
    wig::World& Wd = b->hw[world];
    const uint64_t bytes = b->pooled ? persistent_bytes(b->L[world])
                                     : world_buffers_bytes(b->L[world]) + scratch_bytes(Wd.D);
    void* p = nullptr;
    if (cudaMallocAsync(&p, bytes, s) != cudaSuccess) {
        cudaGetLastError();
        return fail(WIG_E_OOM, "device memory for the world");
    }
    CUDA_TRY(cudaMemsetAsync(p, 0, bytes, s));
    char* q = static_cast<char*>(p);
    for (int w = 0; w < 7; w++) {
        if (b->pooled && borrowed(w)) {
            *buffer_slot(Wd.D, w) = nullptr;  // the lane's pool at each step
            continue;
        }
        *buffer_slot(Wd.D, w) = q;
        q += align256(b->pooled ? persistent_buffer_bytes(b->L[world], w) : buffer_bytes(b->L[world], w));
    }
    if (!b->pooled) scratch_take(Wd, q, b->S.coarse_cells);
    CUDA_TRY(cudaMemcpyAsync(b->d_worlds + world, &Wd, sizeof(wig::World), cudaMemcpyHostToDevice, s));
    for (auto& ln : b->lane)
        if (ln.d_table) CUDA_TRY(cudaMemcpyAsync(ln.d_table + world, &Wd, sizeof(wig::World), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    b->wmem[world] = p;
    b->resident += bytes;
    b->bound[world] = 1;
    b->dirty[world] = 1;  // (its tiling parity carries on from its last step)
    return WIG_OK;
}

int wig_batch_evict(wig_batch* b, uint32_t world, void* stream) {
    if (!b) return fail(WIG_E_ARG, "null batch");
    if (world >= b->K) return fail(WIG_E_ARG, "world index out of range");
    if (b->wmem.empty() || !b->wmem[world]) return fail(WIG_E_STATE, "world not admitted");
    cudaStream_t s = (cudaStream_t)stream;
    // its last step done before its memory goes back to the pool
    if (b->stepped_on[world] != s) CUDA_TRY(cudaStreamSynchronize(b->stepped_on[world]));
    wig::World& Wd = b->hw[world];
    const uint64_t bytes = b->pooled ? persistent_bytes(b->L[world])
                                     : world_buffers_bytes(b->L[world]) + scratch_bytes(Wd.D);
    CUDA_TRY(cudaFreeAsync(b->wmem[world], s));
    for (int w = 0; w < 7; w++) *buffer_slot(Wd.D, w) = nullptr;
    b->wmem[world] = nullptr;
    b->resident -= bytes;
    b->bound[world] = 0;
    return WIG_OK;
}

uint64_t wig_batch_resident_bytes(const wig_batch* b) { return b ? b->resident : 0u; }

int wig_batch_world_bytes_split(const wig_world_desc* d, uint64_t* persistent, uint64_t* transient) {
    if (!persistent || !transient) return fail(WIG_E_ARG, "null argument");
    wig_world_layout L;
    int rc = layout_of(d, &L);
    if (rc) return rc;
    wig::Dev D{};
    dev_shape(D, L);
    *persistent = persistent_bytes(L);
    *transient = transient_bytes(L, D);
    return WIG_OK;
}

int wig_batch_set_launch(wig_batch* b, uint32_t knob, uint32_t value) {
    if (!b) return fail(WIG_E_ARG, "null batch");
    if (knob >= WIG_LAUNCH_KNOBS) return fail(WIG_E_ARG, "unknown launch knob");
    // a single world's coarse levels may start higher: on a cluster
    const uint32_t most = knob != WIG_LAUNCH_COARSE_CELLS ? 64u
                          : b->K == 1                    ? wig::COARSE_CLUSTER_CELLS
                                                         : wig::COARSE_CTA_CELLS;
    if (value < 1u || value > most) return fail(WIG_E_ARG, "launch knob value out of range");
    CUDA_TRY(cudaDeviceSynchronize());
    wig::BatchShape& S = b->S;
    switch (knob) {
    case WIG_LAUNCH_COARSE_CELLS: {
        const uint32_t was = S.coarse_cells;
        S.coarse_cells = value;
        level_shape(b);
        if (S.coarse_smem > 220u * 1024u || wig::fast_prepare_attributes(S.coarse_smem) != cudaSuccess) {
            S.coarse_cells = was;
            level_shape(b);
            return fail(WIG_E_ARG, "coarse levels too large for the coarse kernel");
        }
        CUDA_TRY(cudaMemcpy(b->d_worlds, b->hw.data(), sizeof(wig::World) * b->K, cudaMemcpyHostToDevice));
        break;
    }
    case WIG_LAUNCH_LEVEL_PER_SM: S.level_per_sm = value; break;
    case WIG_LAUNCH_CG_PER_SM: S.cg_per_sm = value; break;
    default: S.relax_per_sm = value; break;
    }
    for (auto& ln : b->lane) drop_graphs(ln);
    return WIG_OK;
}

int wig_batch_get_launch(const wig_batch* b, uint32_t knob, uint32_t* value) {
    if (!b || !value) return fail(WIG_E_ARG, "null argument");
    switch (knob) {
    case WIG_LAUNCH_COARSE_CELLS: *value = b->S.coarse_cells; break;
    case WIG_LAUNCH_LEVEL_PER_SM: *value = b->S.level_per_sm; break;
    case WIG_LAUNCH_CG_PER_SM: *value = b->S.cg_per_sm; break;
    case WIG_LAUNCH_RELAX_PER_SM: *value = b->S.relax_per_sm; break;
    default: return fail(WIG_E_ARG, "unknown launch knob");
    }
    return WIG_OK;
}

int wig_batch_set_lane_pool(wig_batch* b, uint32_t lane, uint64_t bytes) {
    if (!b) return fail(WIG_E_ARG, "null batch");
    if (lane >= WIG_BATCH_LANES) return fail(WIG_E_ARG, "lane out of range");
    if (b->wmem.empty()) return fail(WIG_E_STATE, "not a deferred batch");
    for (uint32_t k = 0; k < b->K; k++)
        if (b->wmem[k]) return fail(WIG_E_STATE, "set the pools before admitting worlds");
    Lane& ln = b->lane[lane];
    CUDA_TRY(cudaDeviceSynchronize());
    if (ln.d_pool) { cudaFree(ln.d_pool); ln.d_pool = nullptr; ln.pool_bytes = 0; }
    if (cudaMalloc(&ln.d_pool, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(WIG_E_OOM, "cudaMalloc of a lane pool");
    }
    ln.pool_bytes = bytes;
    if (!ln.d_table) {
        if (cudaMalloc(&ln.d_table, sizeof(wig::World) * b->K) != cudaSuccess) return fail(WIG_E_OOM, "cudaMalloc lane table");
        CUDA_TRY(cudaMemcpy(ln.d_table, b->hw.data(), sizeof(wig::World) * b->K, cudaMemcpyHostToDevice));
    }
    ln.Bt.worlds = ln.d_table;
    ln.ctl.table = ln.d_table;
    ln.ctl.entries = reinterpret_cast<const wig::World*>(ln.d_up + b->entries_at);
    drop_graphs(ln);
    b->pooled = true;
    return WIG_OK;
}

}  // extern "C"
