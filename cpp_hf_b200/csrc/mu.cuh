// Internal interface of the chemical-potential solvers.
#pragma once

#include "common.cuh"

namespace cpphf {

size_t mu_workspace_bytes(int64_t nk, int64_t nb);
// mode 0: find_mu_bisection (raw weights, target n_e; mu0, when given and
// finite, warm-starts the root the bisection levels are replayed against, with
// the same result), mode 1: solve_mu_inloop (normalised weights, warm start *mu0).  Writes *mu_out (NaN on a device wait
// timeout).
int mu_solve(const double* eps, const double* w, int64_t nk, int64_t nb, double target,
             const double* mu0, double T, int maxiter, int mode, double* mu_out, void* ws,
             size_t wsb, cudaStream_t st);

}  // namespace cpphf
