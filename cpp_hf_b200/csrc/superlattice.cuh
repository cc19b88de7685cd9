// Internal interface of the superlattice Fock terms (superlattice.cu).
#pragma once

#include "common.cuh"

namespace cpphf {

size_t superlattice_workspace_bytes(int64_t n_pairs, int64_t nG, int64_t orb, int64_t NX, int64_t NY, int orbital_vr);
int superlattice_streamed(const double2* rho, const double2* VR, const double2* VRo, const int64_t* g_a_off,
                          const int64_t* pair_i, const int64_t* pair_j, const int64_t* pair_start, int64_t n_delta,
                          int64_t nkx, int64_t nky, int64_t nG, int64_t orb, int64_t NX, int64_t NY, int hermitian,
                          double2* sigma, void* ws, size_t wsb, cudaStream_t st);
size_t sl_hartree_workspace_bytes(const cpphf_superlattice* sl);
// k-independent superlattice Hartree from rho_bar (nb x nb) into SC (added when accumulate)
int sl_hartree(const cpphf_superlattice* sl, const double2* rho_bar, double2* SC, int accumulate, void* ws,
               cudaStream_t st);
// out = a - b over n complex elements
int field_diff(const double2* a, const double2* b, double2* out, int64_t n, cudaStream_t st);

}  // namespace cpphf
