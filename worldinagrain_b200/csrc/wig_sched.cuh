// wig_sched.cuh — writing a batch's work lists on the device.
#pragma once
#include "wig_passes.cuh"

namespace wig {

// The schedule's device arrays: the step's subset of worlds (nsub entries of
// sub, world-table indices) with their heads (null: the worlds' StepStates
// are already written), each list's first item per subset entry (off, list
// L at L * (max_worlds + 1)), and the lists themselves (writable views of
// Batch::items and Batch::count).
struct SchedCtl {
    const uint32_t* nsub;
    const uint32_t* sub;
    const StepHead* heads;
    uint32_t* off;
    uint32_t* items;
    uint32_t* count;
    uint32_t max_worlds;
    // pooled batches: the stepping worlds' table entries for this step (their
    // per-step memory in the lane's pool), copied into the lane's table
    const World* entries;
    World* table;
};

// Writes the lists of one point of a step: phase 0 at its start (WB, PS,
// ONE_ALL, ONE, RES, SM; and the worlds' StepStates from the heads, and in
// a pooled batch their table entries), phase 1 after compact (ACT, RET,
// ACT4, RELAX, PP).  Two launches on stream s.
void sched_lists(const Batch& Bt, const SchedCtl& c, const BatchShape& S, int phase, cudaStream_t s);

}  // namespace wig
