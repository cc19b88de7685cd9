// Helpers shared by the solver loops (solver.cu, rtr.cu).
#pragma once

#include "common.cuh"

namespace cpphf {

// grid of a flat grid-stride kernel: enough blocks for n items, at most 8 per SM
unsigned grid_for(int64_t n, int threads);
// Page-locked scratch for the solver loops' scalar read-backs, kHostScalars
// doubles per host thread, allocated on the thread's first call and kept until
// it exits (a pageable array if the allocation fails).  Copies into it queue as
// asynchronous DMA behind the stream's work, so the reads of one loop step cost
// one stream synchronize.  A solve fetches it before any graph capture.
constexpr int kHostScalars = 64;
double* host_scalars();
// dst = (src + src^H) / 2 per k-point (src may alias dst)
int hermitize(const double2* src, double2* dst, int64_t nk, int nb, cudaStream_t st);
// apply a solver projector to a device field; a non-zero return becomes an error
int call_project(cpphf_project_fn fn, void* user, double2* M, const cpphf_kernel* K, cudaStream_t st);
// out = w / wsum
int scale_weights(const double* w, double wsum, double* out, int64_t n, cudaStream_t st);

}  // namespace cpphf
