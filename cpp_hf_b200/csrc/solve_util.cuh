// Helpers shared by the solver loops (solver.cu, rtr.cu).
#pragma once

#include "common.cuh"

namespace cpphf {

// grid of a flat grid-stride kernel: enough blocks for n items, at most 8 per SM
unsigned grid_for(int64_t n, int threads);
// dst = (src + src^H) / 2 per k-point (src may alias dst)
int hermitize(const double2* src, double2* dst, int64_t nk, int nb, cudaStream_t st);
// apply a solver projector to a device field; a non-zero return becomes an error
int call_project(cpphf_project_fn fn, void* user, double2* M, const cpphf_kernel* K, cudaStream_t st);
// out = w / wsum
int scale_weights(const double* w, double wsum, double* out, int64_t n, cudaStream_t st);

}  // namespace cpphf
