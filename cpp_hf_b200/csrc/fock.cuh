// Internal interface of the Fock assembly.
#pragma once

#include "common.cuh"

namespace cpphf {

int validate_kernel(const cpphf_kernel* K);
size_t build_fock_workspace_bytes(const cpphf_kernel* K);
// Sigma, F fields; hd_out (nb) may be null; energy (device scalar) may be null;
// Hdense may be null.
int build_fock(const cpphf_kernel* K, const double2* P, double2* Sigma, double2* F, double* hd_out,
               double* energy, double2* Hdense, void* ws, size_t wsb, cudaStream_t st);

}  // namespace cpphf
