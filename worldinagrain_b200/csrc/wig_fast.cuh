// wig_fast.cuh — the fast form of the pressure solve: the same arithmetic as
// the reference's CG / V-cycle passes (fluid.wgsl:2047-2893), over
// structure-of-arrays scratch with the stencil's coefficients worked out once
// a step, its iterations looped on the device by a CUDA-graph WHILE node, one
// launch a pass for all the worlds of a batch.
#pragma once
#include "wig_passes.cuh"

namespace wig {

// One world's fast form with its step's settings: the persistent solve's
// argument (a batch of one world).
struct Fast : FastW {
    Dev D;
    uint32_t solve_grid;       // CTAs of the persistent solve (all resident)
    uint32_t max_cycles;
};

// The one-CTA coarse kernel holds levels of at most this many cells; CTA 0
// of the persistent solve, of at most PERSISTENT_CTA_CELLS.
constexpr uint32_t COARSE_CTA_CELLS = 4096;
// A single world's coarse levels from a level of up to this many cells run
// on a thread-block cluster (k_fCoarseCluster).
constexpr uint32_t COARSE_CLUSTER_CELLS = 16384;

// A world's first level of at most `cells` cells (its coarsest when none
// above it is): where the coarse kernel takes over.
inline uint32_t coarse_level(const Dev& D, uint32_t cells) {
    for (uint32_t l = 1; l <= D.levels; l++)
        if ((size_t)D.level_w[l] * D.level_h[l] <= cells) return l;
    return D.levels;
}
constexpr uint32_t PERSISTENT_CTA_CELLS = 1024;

// A profiler's hook around each launch: fn(ctx, slot, 0) before, (ctx, slot, 1) after.
struct Marker {
    void (*fn)(void* ctx, int slot, int phase);
    void* ctx;
};

// While an iteration is captured into the loop's body graph: a stream for
// the bodies of the conditional nodes inside it (the mixed form's
// true-residual check and fix run in IF nodes, so the iterations that need
// neither launch neither), and the first CUDA error met.
struct NestCapture {
    cudaStream_t s;
    cudaError_t err;
};

// Launchers over a batch (stream-ordered; all capturable).  `one`: the
// batch's only world (host copy), passed to the kernels as a parameter; null
// for a batch of several.  fast_cycle returns the launches every iteration
// makes; `nest`: the capture's stream for conditional bodies (null when
// launched eagerly: the check and the fix are then launched every
// iteration and return at once when not needed).
void fast_setup(const Batch& Bt, const BatchShape& S, const World* one, cudaStream_t s, const Marker* m);
uint32_t fast_cycle(const Batch& Bt, const BatchShape& S, const World* one, cudaStream_t s, const Marker* m,
                    NestCapture* nest = nullptr);
// cgFinish; `two_p`: the fast form's p is in P or P2 by the iterations' parity.
void fast_finish(const Batch& Bt, const BatchShape& S, const World* one, bool two_p, cudaStream_t s, const Marker* m);
// Level 0's arrays of one world zeroed (after its buffers are written by the host).
void fast_zero_level0(const FastW& F, uint32_t cells, cudaStream_t s);
// The same for the blocks not worked on, of every world of the step whose
// scratch a pool lends (after compact).
void fast_zero_idle(const Batch& Bt, const BatchShape& S, cudaStream_t s);
// Shared memory of the coarse kernel for a world, and the kernel's limit set.
size_t fast_coarse_smem(const Dev& D, uint32_t lc);
// Shared memory a CTA of the cluster coarse kernel takes for a single world
// from level lc; 0 when that kernel does not apply (level lc fits the one-CTA
// kernel, or the world's coarsest level does not fit one CTA of the cluster).
size_t fast_cluster_smem(const Dev& D, uint32_t lc);
cudaError_t fast_prepare_attributes(size_t smem);
// The persistent solve of one world: all iterations in one cooperative launch.
size_t fast_solve_smem(const Fast& F);
cudaError_t fast_solve_grid(const Fast& F, uint32_t* grid);
cudaError_t fast_solve(const Fast& F, bool shifted, cudaStream_t s, const Marker* m);

}  // namespace wig
