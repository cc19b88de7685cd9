// Internal interface of the exchange (FFT convolution) kernels.
#pragma once

#include "common.cuh"

namespace cpphf {

struct ExchangeGeom {
    int n0, n1;  // mesh (nk1, nk2)
    int nb;      // orbitals
    int C;       // channels transformed: nb*nb, or nb*(nb+1)/2 with HCP
    int dv;      // VR channel width: 1 (scalar broadcast) or nb*nb (elementwise)
    int Ct;      // channel stride of the intermediate T
    int hcp;     // upper-triangle packing with conjugate mirror on unpack
    int shift;   // apply ifftshift on (kx, ky) to the output
    unsigned* err = nullptr;  // device error word for bounded waits
};

size_t exchange_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb, int hcp, int precision);

// Sigma = -IFFT2[FFT2(P - refP) * VR]; refP may be null; Sigma may alias P.
int exchange(const double2* P, const double2* refP, const double2* VR, double2* Sigma, int64_t nk1,
             int64_t nk2, int64_t nb, int64_t dv, int hcp, int shift, int precision,
             void* workspace, size_t workspace_bytes, cudaStream_t st);

// The columns pass alone on an (n0, n1, g.C) field T (complex128, or complex64
// with precision 32): FFT along kx, times VR (g.dv = 1: one scalar per q,
// else g.dv = g.C channels laid out like T), inverse FFT along kx, in place.
int exchange_columns(void* T, const double2* VR, const ExchangeGeom& g, int precision, cudaStream_t st);

}  // namespace cpphf
