// Internal interface of the trust-region Newton solver (rtr.cu).
#pragma once

#include "common.cuh"

namespace cpphf {

size_t solve_rtr_workspace_bytes(const cpphf_kernel* K, const cpphf_dm_config* cfg);
int solve_rtr(const cpphf_kernel* K, const cpphf_dm_config* cfg, const double2* P0, double n_e,
              cpphf_project_fn project, void* puser, double2* Q_out, double* p_out, double2* D_out, double2* F_out,
              double* hist_E, double* hist_G, cpphf_dm_result* res, void* ws, size_t wsb, cudaStream_t st);

}  // namespace cpphf
