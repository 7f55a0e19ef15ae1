// wig_passes.cuh — launchers of the liquid step's pass kernels.
#pragma once
#include "wig_device.cuh"

namespace wig {

// Host-side shape of a batch: the most items each work list can hold (grid
// sizes of the kernels over it).
struct BatchShape {
    uint32_t max_items[L_COUNT];
    uint32_t worlds;
    uint32_t levels;       // deepest coarse level of any world
    uint32_t lc_max;       // deepest level any world restricts by itself
    size_t coarse_smem;    // the coarse kernel's shared memory for the largest world (a CTA's, on a cluster)
    uint32_t cluster;      // a single world's coarse levels on a thread-block cluster
    // launch shapes (wig_launch_knob): none changes a result
    uint32_t coarse_cells;  // the coarse kernel from a world's first level of at most this many cells
    uint32_t level_per_sm, cg_per_sm, relax_per_sm;
};

// CTAs for a kernel over list `list` with `per_sm` CTAs a multiprocessor.
unsigned list_grid(const BatchShape& S, uint32_t list, unsigned per_sm);

// One reference pass (enum wig_pass) at Level (level, cycle), on stream s:
// over the batch's work lists, or (the plain form's solve passes) over
// world 0, whose descriptor D0 is.
int launch_pass(const Batch& Bt, const BatchShape& S, const Dev& D0, int pass, uint32_t level, uint32_t cycle,
                cudaStream_t s);
// The fast forms' cgStart + cgJoin: part 0 cgStart with each block's own
// labelling (k_cgStartLocal), part 1 the joins between blocks; the same
// regions and roots as the two passes.
void launch_labels(const Batch& Bt, const BatchShape& S, cudaStream_t s, int part);
// The plain form's tolerance norms on world 0: which 0 = ||b||^2 after
// cgResidual, 1 = ||r||/||b|| after cgUpdate.
int launch_norm(const Dev& D, int which, uint32_t cycle, cudaStream_t s);
}  // namespace wig
