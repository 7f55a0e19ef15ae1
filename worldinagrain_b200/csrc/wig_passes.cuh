// wig_passes.cuh — launchers of the liquid step's pass kernels.
#pragma once
#include "wig_device.cuh"

namespace wig {
// One reference pass (enum wig_pass) at Level (level, cycle), on stream s.
int launch_pass(const Dev& D, int pass, uint32_t level, uint32_t cycle, cudaStream_t s);
// The tolerance form's norms: which 0 = ||b||^2 after cgResidual, 1 = ||r||/||b|| after cgUpdate.
int launch_norm(const Dev& D, int which, uint32_t cycle, cudaStream_t s);
}  // namespace wig
