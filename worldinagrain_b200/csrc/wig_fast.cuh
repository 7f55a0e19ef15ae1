// wig_fast.cuh — the fast form of the pressure solve: the same arithmetic as
// the reference's CG / V-cycle passes (fluid.wgsl:2047-2893), over
// structure-of-arrays scratch with the stencil's coefficients worked out once
// a step, its iterations looped on the device by a CUDA-graph WHILE node.
#pragma once
#include "wig_device.cuh"

namespace wig {

// One multigrid level's arrays, a float per cell (row-major, the level's
// width): potentials and right-hand sides (pressure x, drift y), density,
// and the stencil's coefficients to the left, right, upper and lower
// neighbours (0 past an obstacle or the edge) with their sum.
struct Lvl {
    float *px, *py, *rx, *ry, *rho;
    float *b0, *b1, *b2, *b3, *diag;
};

struct Fast {
    Dev D;
    Lvl L[WIG_MG_LEVELS + 1];  // level 0 (the cells) .. D.levels
    float* pin;                // level 0: PIN at a pinned root, else 0
    uint8_t* fmask;            // level 0: bit d set when neighbour d is liquid
    float *rimx, *rimy;        // level 0: the relaxation's rim snapshot
    float *X, *R, *P, *Q;      // level 0: CG's x, r, p, A p
    float* part32;             // 2 per block
    double* part64;            // 2 per block
    uint32_t lc;               // first level the one-CTA kernel solves (the multi-kernel form)
    uint32_t lp;               // first level CTA 0 of the persistent solve holds (<= 1024 cells)
    uint32_t solve_grid;       // CTAs of the persistent solve (all resident)
    uint32_t max_cycles;
    unsigned long long cond;   // cudaGraphConditionalHandle of the iteration loop (0: none, a host-driven loop)
};

// The one-CTA coarse kernel holds levels of at most this many cells; CTA 0
// of the persistent solve, of at most PERSISTENT_CTA_CELLS.
constexpr uint32_t COARSE_CTA_CELLS = 4096;
constexpr uint32_t PERSISTENT_CTA_CELLS = 1024;

// A profiler's hook around each launch: fn(ctx, slot, 0) before, (ctx, slot, 1) after.
struct Marker {
    void (*fn)(void* ctx, int slot, int phase);
    void* ctx;
};

// Launchers (stream-ordered; all capturable).  fast_cycle returns its launches.
void fast_setup(const Fast& F, cudaStream_t s, const Marker* m);
uint32_t fast_cycle(const Fast& F, bool shifted, cudaStream_t s, const Marker* m);
void fast_finish(const Fast& F, cudaStream_t s, const Marker* m);
void fast_zero_level0(const Fast& F, cudaStream_t s);
cudaError_t fast_prepare_attributes(size_t smem);
size_t fast_coarse_smem(const Fast& F);
// the persistent solve: all iterations in one cooperative launch
size_t fast_solve_smem(const Fast& F);
cudaError_t fast_solve_grid(const Fast& F, uint32_t* grid);
cudaError_t fast_solve(const Fast& F, bool shifted, cudaStream_t s, const Marker* m);

}  // namespace wig
