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

constexpr int kFockMaxPartials = 2048;  // energy partials of the assembly launches

// Hermitian-packed Fock build (fock_packed.cu).  Active for a kernel with
// hermitian_packing set, nb <= 8, VR of width 1 or nb, no superlattice terms
// and mesh axes with a pipelined codelet.  The Sigma field is written only
// when Sigma != null (the solvers do not need it).
struct PackGeom {
    int nb, nchunk, CB, CBp, Ct;  // chunks of row pairs, nb + 1 channels each, CBp slots, Ct slots in all
};
bool packed_fock_eligible(const cpphf_kernel* K);
size_t packed_field_bytes(const cpphf_kernel* K);
size_t packed_fock_workspace_bytes(const cpphf_kernel* K);
int pack_kernel_fields(const cpphf_kernel* K, double2* VRp, double2* hp, cudaStream_t st);
int build_fock_packed(const cpphf_kernel* K, const double2* P, double2* Sigma, double2* F, const double* hd,
                      const double2* SC, const double2* rho_bar, double* energy, double2* Hdense, double* part,
                      unsigned* counter, void* ws, size_t wsb, cudaStream_t st);
// Solvers: bytes for the packed VR / h a kernel lacks (0 when the packed build
// cannot run), and a copy of K with them made in `ws` (once per solve).
size_t solver_pack_bytes(const cpphf_kernel* K);
int solver_pack(const cpphf_kernel* K, cpphf_kernel* out, void* ws, cudaStream_t st);
// build_fock workspace bytes for K once its packed fields exist.
size_t fock_bytes_packed_kernel(const cpphf_kernel* K);
// The Sigma a solver passes to build_fock: none when the packed build runs.
inline double2* solver_sigma(const cpphf_kernel* K, double2* Sig) { return packed_fock_eligible(K) ? nullptr : Sig; }

}  // namespace cpphf
