// wig_api.cu — the C ABI (include/wig_fluid.h): world handles, bound
// buffers, and the step driver that replaces Simulation.encodeFluid
// (js/sim.js:2466-2612).
//
// A step is the reference's pass sequence, recorded once per shape (max
// cycles, flags, the tiling parity it starts on) into a CUDA graph and
// replayed: the per-step inputs (the Params uniform) reach the device as one
// small copy from pinned host memory ahead of the graph, and the report words
// come back as one small copy after it, the reference's writeBuffer and
// mapped report buffer (js/sim.js:1975-1995, :1763, :1882-1900).

#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "wig_device.cuh"
#include "wig_fast.cuh"
#include "wig_passes.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace

namespace wig {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace wig

namespace {

#define CUDA_TRY(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(WIG_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device-side report: the FLUID_COUNT words, the particle count and the
// solve's residuals, gathered by k_report at the end of a step.
struct Report {
    uint32_t count[WIG_FLUID_STATS];
    uint32_t particles;
    uint32_t err;
    uint32_t pad;
    double rel;
    double bnorm2;
};

__global__ void k_report(wig::Dev D, Report* out) {
    if (threadIdx.x == 0) {
        for (uint32_t k = 0; k < WIG_FLUID_STATS; k++) out->count[k] = D.blocks[4u * D.B + k];
        out->particles = D.sorted[0];
        out->err = D.st->err;
        out->rel = D.st->rel;
        out->bnorm2 = D.st->bnorm2;
    }
}

constexpr int RING = 8;

}  // namespace

struct wig_fluid {
    wig_world_layout L{};
    wig::Dev D{};
    int device = 0;
    void* own[7] = {nullptr};
    bool bound = false;
    wig_elem* d_elems = nullptr;
    wig::StepState* d_st = nullptr;
    wig::StepState* h_st = nullptr;  // pinned ring of RING
    cudaEvent_t st_ev[RING] = {};
    int st_at = 0;
    Report* d_report = nullptr;
    Report* h_report = nullptr;      // pinned
    double* d_part64 = nullptr;
    double* d_norm64 = nullptr;
    bool shifted_first = false;
    cudaStream_t cap = nullptr;      // capture stream
    cudaStream_t last_stream = nullptr;
    std::map<uint64_t, std::pair<cudaGraph_t, cudaGraphExec_t>> graphs;
    std::map<uint64_t, uint32_t> graph_launches;  // kernels in each graph (fast form: outside the loop)
    std::map<uint64_t, uint32_t> graph_body;      // fast form: kernels per iteration
    uint32_t last_launches = 0;
    uint32_t last_body = 0;
    uint32_t last_cycles_flags = 0;
    // the fast form's scratch
    wig::Fast F{};
    void* fast_mem = nullptr;
    bool fast_dirty = true;
    cudaStream_t cap2 = nullptr;     // capture stream of the iteration loop's body
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
    uint64_t cap = d->capacity ? d->capacity : (uint64_t)((double)C * L->liquid_per_cell * 1.25 + 0.999999);
    if (!d->capacity) {
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

void** buffer_slot(wig_fluid* h, int which) {
    switch (which) {
    case 0: return (void**)&h->D.cells;
    case 1: return (void**)&h->D.sorted;
    case 2: return (void**)&h->D.parts;
    case 3: return (void**)&h->D.counters;
    case 4: return (void**)&h->D.field;
    case 5: return (void**)&h->D.blocks;
    case 6: return (void**)&h->D.cg;
    default: return nullptr;
    }
}

void drop_graphs(wig_fluid* h) {
    for (auto& kv : h->graphs) {
        if (kv.second.second) cudaGraphExecDestroy(kv.second.second);
        if (kv.second.first) cudaGraphDestroy(kv.second.first);
    }
    h->graphs.clear();
    h->graph_launches.clear();
    h->graph_body.clear();
}

// Writes this step's state into the next pinned slot and copies it to the
// device on stream s.
int push_state(wig_fluid* h, const wig_params* P, uint32_t flags, double tol, cudaStream_t s, bool params_only) {
    int k = h->st_at;
    h->st_at = (h->st_at + 1) % RING;
    CUDA_TRY(cudaEventSynchronize(h->st_ev[k]));
    wig::StepState* st = h->h_st + k;
    std::memset(st, 0, sizeof(*st));
    st->P = *P;
    st->P.size[0] = h->L.width;
    st->P.size[1] = h->L.height;
    st->tol_mode = (flags & WIG_STEP_TOLERANCE) ? 1u : 0u;
    st->f64 = (flags & WIG_STEP_F64_DOTS) ? 1u : 0u;
    st->tol = tol;
    st->rel = 1.0;
    size_t bytes = params_only ? sizeof(wig_params) : sizeof(wig::StepState);
    CUDA_TRY(cudaMemcpyAsync(h->d_st, st, bytes, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaEventRecord(h->st_ev[k], s));
    return WIG_OK;
}

// Per-pass timing of an eagerly launched step (the reference's per-phase
// GPU timestamps, js/timer.js:7-98): events around each launch.
struct Prof {
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
};

// Launch recording with optional per-launch events (Prof).
struct Rec {
    wig_fluid* h;
    cudaStream_t s;
    Prof* prof;
    uint32_t launches = 0;
    cudaEvent_t pending = nullptr;
    template <class Fn>
    void timed(int id, Fn fn) {
        cudaEvent_t a = nullptr, b = nullptr;
        if (prof) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, s);
        }
        fn();
        launches++;
        if (prof) {
            cudaEventRecord(b, s);
            prof->marks.push_back({id, {a, b}});
        }
    }
    void run(int pass, uint32_t level = 0, uint32_t cycle = 0) {
        timed(pass, [&] { wig::launch_pass(h->D, pass, level, cycle, s); });
    }
    void norm(int which, uint32_t cycle) {
        timed(WIG_SLOT_NORM, [&] { wig::launch_norm(h->D, which, cycle, s); });
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

// encodeFluid's passes before the solve (js/sim.js:2486-2521).
void record_pre(Rec& R, uint32_t flags) {
    R.run(WIG_PASS_SYNC);
    R.run(WIG_PASS_SYNC_PARTICLES);
    R.run(WIG_PASS_SYNC_SEED);
    R.run(WIG_PASS_COMPACT);
    R.run(WIG_PASS_RETIRE);
    R.run(WIG_PASS_CLEAR);
    R.run(WIG_PASS_GATHER);
    R.run(WIG_PASS_SEAL_JOIN);
    R.run(WIG_PASS_SEAL_ANCHOR);
    R.run(WIG_PASS_CLASSIFY);
    R.run(WIG_PASS_SET_FACES);
    if (flags & WIG_STEP_VISCOUS)
        for (int i = 0; i < 8; i++) {
            R.run(WIG_PASS_VISCOSITY_RED);
            R.run(WIG_PASS_VISCOSITY_BLACK);
        }
    R.run(WIG_PASS_UNPRESS);
    R.run(WIG_PASS_DIVERGENCE);
}

// encodeFluid's passes after the solve (js/sim.js:2592-2611) and the report.
void record_post(Rec& R) {
    R.run(WIG_PASS_PROJECT);
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
    R.timed(WIG_SLOT_REPORT, [&] { k_report<<<1, 32, 0, R.s>>>(R.h->D, R.h->d_report); });
}

// Records the plain form's step (one kernel per reference pass, every
// iteration encoded) on stream s; returns the number of kernels launched.
uint32_t record_step(wig_fluid* h, uint32_t max_cycles, uint32_t flags, bool shifted, cudaStream_t s, Prof* prof) {
    Rec R{h, s, prof};
    const bool tol = (flags & WIG_STEP_TOLERANCE) != 0u;
    if (flags & WIG_STEP_BOOKKEEPING_ONLY) {
        R.run(WIG_PASS_SYNC_MARKS);
        R.run(WIG_PASS_COMPACT);
        R.run(WIG_PASS_RETIRE);
        R.timed(WIG_SLOT_REPORT, [&] { k_report<<<1, 32, 0, s>>>(h->D, h->d_report); });
        return R.launches;
    }
    record_pre(R, flags);
    const uint32_t deepest = h->L.levels;
    R.run(WIG_PASS_CG_START);
    R.run(WIG_PASS_CG_JOIN);
    R.run(WIG_PASS_CG_ANCHOR);
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
        R.run(WIG_PASS_CG_APPLY, 0, cycle);
        R.run(WIG_PASS_CG_ALPHA, 0, cycle);
        R.run(WIG_PASS_CG_UPDATE, 0, cycle);
        if (tol) R.norm(1, cycle);
    }
    R.run(WIG_PASS_CG_FINISH);
    record_post(R);
    return R.launches;
}

wig::Fast fast_of(wig_fluid* h, uint32_t max_cycles, unsigned long long cond) {
    wig::Fast F = h->F;
    F.D = h->D;
    F.max_cycles = max_cycles;
    F.cond = cond;
    return F;
}

// Records the fast form's step.  With `capture`, s is capturing into a graph
// and the iterations become a WHILE node whose body is captured on h->cap2;
// else the iterations are launched from the host, each decided by reading
// back the device's verdict (the profiler's path).  *outside gets the kernels
// outside the loop (all of them when not capturing), *body those of one
// iteration of the loop.
int record_step_fast(wig_fluid* h, uint32_t max_cycles, uint32_t flags, bool shifted, cudaStream_t s, Prof* prof,
                     bool capture, uint32_t* outside, uint32_t* body) {
    Rec R{h, s, prof};
    record_pre(R, flags);
    R.run(WIG_PASS_CG_START);
    R.run(WIG_PASS_CG_JOIN);
    R.run(WIG_PASS_CG_ANCHOR);
    wig::Marker mk{&Rec::mark, &R};
    const wig::Fast F0 = fast_of(h, max_cycles, 0ull);
    wig::fast_setup(F0, s, prof ? &mk : nullptr);
    R.launches++;
    if (flags & WIG_STEP_PERSISTENT) {
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
        CUDA_TRY(cudaStreamBeginCaptureToGraph(h->cap2, bodyGraph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        const wig::Fast F = fast_of(h, max_cycles, (unsigned long long)handle);
        *body = wig::fast_cycle(F, shifted, h->cap2, nullptr);
        cudaGraph_t captured = nullptr;
        CUDA_TRY(cudaStreamEndCapture(h->cap2, &captured));
    } else {
        uint32_t* cont = &h->h_report->pad;
        for (uint32_t c = 0; c < max_cycles; c++) {
            R.launches += wig::fast_cycle(F0, shifted, s, prof ? &mk : nullptr);
            CUDA_TRY(cudaMemcpyAsync(cont, &h->d_st->cont, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaStreamSynchronize(s));
            if (!*cont) break;
        }
        *body = 0;
    }
    wig::fast_finish(F0, s, prof ? &mk : nullptr);
    R.launches++;
    record_post(R);
    *outside = R.launches;
    return WIG_OK;
}

bool step_parity(wig_fluid* h, uint32_t flags) {
    if (flags & WIG_STEP_SHIFTED_SET) return (flags & WIG_STEP_SHIFTED_FIRST) != 0u;
    if (!(flags & WIG_STEP_BOOKKEEPING_ONLY)) h->shifted_first = !h->shifted_first;
    return h->shifted_first;
}

}  // namespace

extern "C" {

uint32_t wig_fluid_abi_version(void) { return WIG_ABI_VERSION; }

const char* wig_fluid_last_error(void) { return g_last_error.c_str(); }

int wig_fluid_layout(const wig_world_desc* d, wig_world_layout* out) { return layout_of(d, out); }

int wig_fluid_create(const wig_world_desc* d, const wig_elem* elems, uint32_t n_elems, wig_fluid** out) {
    if (!out) return fail(WIG_E_ARG, "null output handle");
    *out = nullptr;
    if (!elems || n_elems == 0 || n_elems > WIG_MAX_ELEMS) return fail(WIG_E_ARG, "element table empty or too long");
    if (n_elems <= WIG_ELEM_WATER) return fail(WIG_E_ARG, "element table must reach WATER (id 3)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(WIG_E_NO_DEVICE, "no CUDA device");
    }
    wig_fluid* h = new (std::nothrow) wig_fluid();
    if (!h) return fail(WIG_E_OOM, "host allocation failed");
    int rc = layout_of(d, &h->L);
    if (rc) { delete h; return rc; }
    cudaGetDevice(&h->device);
    const wig_world_layout& L = h->L;
    wig::Dev& D = h->D;
    D.W = (int)L.width;
    D.H = (int)L.height;
    D.C = L.cell_count;
    D.F = L.face_count;
    D.B = L.block_count;
    D.BW = L.blocks_wide;
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
    D.n_elems = n_elems;
    auto cleanup = [&](int code, const std::string& m) {
        wig_fluid_destroy(h);
        return fail(code, m);
    };
    if (cudaMalloc(&h->d_elems, sizeof(wig_elem) * n_elems) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMalloc elems");
    if (cudaMemcpy(h->d_elems, elems, sizeof(wig_elem) * n_elems, cudaMemcpyHostToDevice) != cudaSuccess)
        return cleanup(WIG_E_CUDA, "cudaMemcpy elems");
    D.elems = h->d_elems;
    if (cudaMalloc(&h->d_st, sizeof(wig::StepState)) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMalloc step state");
    cudaMemset(h->d_st, 0, sizeof(wig::StepState));
    D.st = h->d_st;
    if (cudaMallocHost(&h->h_st, sizeof(wig::StepState) * RING) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMallocHost");
    for (int k = 0; k < RING; k++)
        if (cudaEventCreateWithFlags(&h->st_ev[k], cudaEventDisableTiming) != cudaSuccess) return cleanup(WIG_E_CUDA, "event");
    if (cudaMalloc(&h->d_report, sizeof(Report)) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMalloc report");
    cudaMemset(h->d_report, 0, sizeof(Report));
    if (cudaMallocHost(&h->h_report, sizeof(Report)) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMallocHost report");
    std::memset(h->h_report, 0, sizeof(Report));
    if (cudaMalloc(&h->d_part64, sizeof(double) * 2 * D.B) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMalloc part64");
    if (cudaMalloc(&h->d_norm64, sizeof(double) * 2 * D.B) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMalloc norm64");
    cudaMemset(h->d_part64, 0, sizeof(double) * 2 * D.B);
    cudaMemset(h->d_norm64, 0, sizeof(double) * 2 * D.B);
    D.part64 = h->d_part64;
    D.norm64 = h->d_norm64;
    if (cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) return cleanup(WIG_E_CUDA, "stream");
    if (cudaStreamCreateWithFlags(&h->cap2, cudaStreamNonBlocking) != cudaSuccess) return cleanup(WIG_E_CUDA, "stream");
    {
        // the fast form's scratch: level 0 (17 floats and a byte a cell), the
        // coarse levels (10 floats a cell), the block partials
        auto align = [](size_t x) { return (x + 255u) & ~(size_t)255u; };
        const size_t C = D.C;
        size_t bytes = align(C) + 17u * align(C * 4u);
        for (uint32_t l = 1; l <= D.levels; l++) bytes += 10u * align((size_t)D.level_w[l] * D.level_h[l] * 4u);
        bytes += align(2u * (size_t)D.B * 4u) + align(2u * (size_t)D.B * 8u);
        if (cudaMalloc(&h->fast_mem, bytes) != cudaSuccess) return cleanup(WIG_E_OOM, "cudaMalloc fast scratch");
        cudaMemset(h->fast_mem, 0, bytes);
        char* p = static_cast<char*>(h->fast_mem);
        auto take = [&](size_t n) { char* q = p; p += align(n); return q; };
        wig::Fast& F = h->F;
        F.fmask = reinterpret_cast<uint8_t*>(take(C));
        auto fl = [&](size_t n) { return reinterpret_cast<float*>(take(n * 4u)); };
        for (uint32_t l = 0; l <= D.levels; l++) {
            const size_t n = l == 0 ? C : (size_t)D.level_w[l] * D.level_h[l];
            wig::Lvl& V = F.L[l];
            V.px = fl(n); V.py = fl(n); V.rx = fl(n); V.ry = fl(n); V.rho = fl(n);
            V.b0 = fl(n); V.b1 = fl(n); V.b2 = fl(n); V.b3 = fl(n); V.diag = fl(n);
        }
        F.pin = fl(C); F.rimx = fl(C); F.rimy = fl(C);
        F.X = fl(C); F.R = fl(C); F.P = fl(C); F.Q = fl(C);
        F.part32 = fl(2u * (size_t)D.B);
        F.part64 = reinterpret_cast<double*>(take(2u * (size_t)D.B * 8u));
        F.lc = D.levels;
        for (uint32_t l = 1; l <= D.levels; l++)
            if ((size_t)D.level_w[l] * D.level_h[l] <= wig::COARSE_CTA_CELLS) { F.lc = l; break; }
        F.lp = D.levels;
        for (uint32_t l = 1; l <= D.levels; l++)
            if ((size_t)D.level_w[l] * D.level_h[l] <= wig::PERSISTENT_CTA_CELLS) { F.lp = l; break; }
        F.D = D;
        size_t smem = wig::fast_coarse_smem(F);
        if (smem > 200u * 1024u) return cleanup(WIG_E_ARG, "coarse levels too large for one CTA");
        if (wig::fast_prepare_attributes(smem) != cudaSuccess) return cleanup(WIG_E_CUDA, "cudaFuncSetAttribute");
        if (wig::fast_solve_grid(F, &F.solve_grid) != cudaSuccess) return cleanup(WIG_E_CUDA, "occupancy of the persistent solve");
        h->fast_dirty = true;
    }
    *out = h;

    return WIG_OK;
}

int wig_fluid_bind(wig_fluid* h, const wig_fluid_buffers* b) {
    if (!h) return fail(WIG_E_ARG, "null handle");
    drop_graphs(h);
    void* given[7] = {nullptr};
    if (b) {
        given[0] = b->cells; given[1] = b->sorted; given[2] = b->parts; given[3] = b->counters;
        given[4] = b->field; given[5] = b->blocks; given[6] = b->cg;
    }
    for (int k = 0; k < 7; k++) {
        void** slot = buffer_slot(h, k);
        if (given[k]) {
            if (((uintptr_t)given[k] & 15u) != 0u) return fail(WIG_E_ARG, "buffer not 16-byte aligned");
            if (h->own[k]) { cudaFree(h->own[k]); h->own[k] = nullptr; }
            *slot = given[k];
        } else if (!h->own[k]) {
            uint64_t bytes = buffer_bytes(h->L, k);
            void* p = nullptr;
            if (cudaMalloc(&p, bytes) != cudaSuccess) {
                cudaGetLastError();
                return fail(WIG_E_OOM, "cudaMalloc of a world buffer failed");
            }
            CUDA_TRY(cudaMemset(p, 0, bytes));
            h->own[k] = p;
            *slot = p;
        }
    }
    h->bound = true;
    h->fast_dirty = true;
    return WIG_OK;
}

int wig_fluid_buffers_of(wig_fluid* h, wig_fluid_buffers* out) {
    if (!h || !out) return fail(WIG_E_ARG, "null argument");
    if (!h->bound) return fail(WIG_E_STATE, "buffers not bound");
    out->cells = h->D.cells; out->sorted = h->D.sorted; out->parts = h->D.parts; out->counters = h->D.counters;
    out->field = h->D.field; out->blocks = h->D.blocks; out->cg = h->D.cg;
    return WIG_OK;
}

int wig_fluid_upload(wig_fluid* h, int which, const void* host, uint64_t offset, uint64_t bytes, void* stream) {
    if (!h || !host) return fail(WIG_E_ARG, "null argument");
    if (!h->bound) return fail(WIG_E_STATE, "buffers not bound");
    uint64_t size = buffer_bytes(h->L, which);
    if (!size || offset > size || bytes > size - offset) return fail(WIG_E_ARG, "upload out of the buffer's range");
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemcpyAsync((char*)*buffer_slot(h, which) + offset, host, bytes, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    h->fast_dirty = true;
    return WIG_OK;
}

int wig_fluid_download(wig_fluid* h, int which, void* host, uint64_t offset, uint64_t bytes, void* stream) {
    if (!h || !host) return fail(WIG_E_ARG, "null argument");
    if (!h->bound) return fail(WIG_E_STATE, "buffers not bound");
    uint64_t size = buffer_bytes(h->L, which);
    if (!size || offset > size || bytes > size - offset) return fail(WIG_E_ARG, "download out of the buffer's range");
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemcpyAsync(host, (const char*)*buffer_slot(h, which) + offset, bytes, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return WIG_OK;
}

int wig_fluid_dispatch(wig_fluid* h, const wig_params* P, int pass, uint32_t level, uint32_t cycle, void* stream) {
    if (!h || !P) return fail(WIG_E_ARG, "null argument");
    if (!h->bound) return fail(WIG_E_STATE, "buffers not bound");
    if (pass < 0 || pass >= WIG_PASS_COUNT) return fail(WIG_E_ARG, "unknown pass");
    if (level > h->L.levels) return fail(WIG_E_ARG, "level past the coarsest");
    cudaStream_t s = (cudaStream_t)stream;
    int rc = push_state(h, P, 0u, 0.0, s, true);
    if (rc) return rc;
    rc = wig::launch_pass(h->D, pass, level, cycle, s);
    if (rc) return fail(rc, "launch");
    CUDA_TRY(cudaGetLastError());
    h->last_stream = s;
    return WIG_OK;
}

int wig_fluid_step(wig_fluid* h, const wig_params* P, uint32_t max_cycles, uint32_t flags, double tolerance, void* stream) {
    if (!h || !P) return fail(WIG_E_ARG, "null argument");
    if (!h->bound) return fail(WIG_E_STATE, "buffers not bound");
    if (max_cycles == 0 || max_cycles > 64) return fail(WIG_E_ARG, "max_cycles out of range (1..64)");
    if ((flags & WIG_STEP_TOLERANCE) && !(tolerance > 0.0)) return fail(WIG_E_ARG, "tolerance must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    const bool sh = step_parity(h, flags);
    int rc = push_state(h, P, flags, tolerance, s, false);
    if (rc) return rc;
    const bool plain = (flags & (WIG_STEP_PLAIN | WIG_STEP_BOOKKEEPING_ONLY)) != 0u;
    if (!plain && h->fast_dirty) {
        wig::fast_zero_level0(fast_of(h, max_cycles, 0ull), s);
        h->fast_dirty = false;
    }
    const uint32_t shape_flags =
        flags & (WIG_STEP_BOOKKEEPING_ONLY | WIG_STEP_VISCOUS | WIG_STEP_TOLERANCE | WIG_STEP_F64_DOTS | WIG_STEP_PLAIN |
                 WIG_STEP_PERSISTENT);
    const uint64_t key = ((uint64_t)max_cycles << 32) | ((uint64_t)shape_flags << 1) | (sh ? 1u : 0u);
    auto it = h->graphs.find(key);
    if (it == h->graphs.end()) {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
        uint32_t n = 0, nb = 0;
        if (plain) {
            n = record_step(h, max_cycles, flags, sh, h->cap, nullptr);
        } else {
            int rc2 = record_step_fast(h, max_cycles, flags, sh, h->cap, nullptr, true, &n, &nb);
            if (rc2) {
                cudaGraph_t junk = nullptr;
                cudaStreamEndCapture(h->cap, &junk);
                if (junk) cudaGraphDestroy(junk);
                return rc2;
            }
        }
        cudaError_t e = cudaStreamEndCapture(h->cap, &g);
        if (e != cudaSuccess) return fail(WIG_E_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ge, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return fail(WIG_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        it = h->graphs.emplace(key, std::make_pair(g, ge)).first;
        h->graph_launches[key] = n;
        h->graph_body[key] = nb;
    }
    h->last_launches = h->graph_launches[key];
    h->last_body = h->graph_body[key];
    CUDA_TRY(cudaGraphLaunch(it->second.second, s));
    if (flags & WIG_STEP_SYNC_STATS) CUDA_TRY(cudaMemcpyAsync(h->h_report, h->d_report, sizeof(Report), cudaMemcpyDeviceToHost, s));
    h->last_stream = s;
    h->last_cycles_flags = flags;
    return WIG_OK;
}

int wig_fluid_step_profile(wig_fluid* h, const wig_params* P, uint32_t max_cycles, uint32_t flags, double tolerance,
                           void* stream, float* ms_out, uint32_t* calls_out) {
    if (!h || !P || !ms_out || !calls_out) return fail(WIG_E_ARG, "null argument");
    if (!h->bound) return fail(WIG_E_STATE, "buffers not bound");
    if (max_cycles == 0 || max_cycles > 64) return fail(WIG_E_ARG, "max_cycles out of range (1..64)");
    if ((flags & WIG_STEP_TOLERANCE) && !(tolerance > 0.0)) return fail(WIG_E_ARG, "tolerance must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    const bool sh = step_parity(h, flags);
    int rc = push_state(h, P, flags, tolerance, s, false);
    if (rc) return rc;
    Prof prof;
    const bool plain = (flags & (WIG_STEP_PLAIN | WIG_STEP_BOOKKEEPING_ONLY)) != 0u;
    h->last_body = 0;
    if (plain) {
        h->last_launches = record_step(h, max_cycles, flags, sh, s, &prof);
    } else {
        if (h->fast_dirty) {
            wig::fast_zero_level0(fast_of(h, max_cycles, 0ull), s);
            h->fast_dirty = false;
        }
        uint32_t n = 0, nb = 0;
        rc = record_step_fast(h, max_cycles, flags, sh, s, &prof, false, &n, &nb);
        if (rc) return rc;
        h->last_launches = n;
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    for (int k = 0; k < WIG_PROFILE_SLOTS; k++) { ms_out[k] = 0.0f; calls_out[k] = 0u; }
    for (auto& m : prof.marks) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, m.second.first, m.second.second);
        ms_out[m.first] += ms;
        calls_out[m.first] += 1u;
        cudaEventDestroy(m.second.first);
        cudaEventDestroy(m.second.second);
    }
    h->last_stream = s;
    return WIG_OK;
}

int wig_fluid_read_stats(wig_fluid* h, wig_fluid_stats* out) {
    if (!h || !out) return fail(WIG_E_ARG, "null argument");
    cudaStream_t s = h->last_stream;
    CUDA_TRY(cudaMemcpyAsync(h->h_report, h->d_report, sizeof(Report), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    const Report& r = *h->h_report;
    std::memset(out, 0, sizeof(*out));
    for (uint32_t k = 0; k < WIG_FLUID_STATS; k++) out->count[k] = r.count[k];
    out->particles = r.particles;
    out->cycles = r.count[WIG_COUNT_CYCLES];
    out->launches = h->last_launches + h->last_body * r.count[WIG_COUNT_CYCLES];
    out->rel_residual = r.rel;
    out->b_norm = r.bnorm2 > 0.0 ? __builtin_sqrt(r.bnorm2) : 0.0;
    if (r.err & wig::ERR_BARRIER) return fail(WIG_E_STATE, "the persistent solve's grid barrier waited past its limit");
    if (r.err) return fail(WIG_E_STATE, "a device loop hit its iteration limit (union-find)");
    if (r.particles > h->L.capacity) return fail(WIG_E_CAPACITY, "more particles than the buffers hold");
    return WIG_OK;
}

void wig_fluid_destroy(wig_fluid* h) {
    if (!h) return;
    if (h->last_stream || true) cudaDeviceSynchronize();
    drop_graphs(h);
    for (int k = 0; k < 7; k++)
        if (h->own[k]) cudaFree(h->own[k]);
    if (h->d_elems) cudaFree(h->d_elems);
    if (h->d_st) cudaFree(h->d_st);
    if (h->h_st) cudaFreeHost(h->h_st);
    for (int k = 0; k < RING; k++)
        if (h->st_ev[k]) cudaEventDestroy(h->st_ev[k]);
    if (h->d_report) cudaFree(h->d_report);
    if (h->h_report) cudaFreeHost(h->h_report);
    if (h->d_part64) cudaFree(h->d_part64);
    if (h->d_norm64) cudaFree(h->d_norm64);
    if (h->cap) cudaStreamDestroy(h->cap);
    if (h->cap2) cudaStreamDestroy(h->cap2);
    if (h->fast_mem) cudaFree(h->fast_mem);
    delete h;
}

}  // extern "C"
