// Internal interface of the trust-region Newton solver (rtr.cu, rtr_small.cu).
#pragma once

#include "common.cuh"

namespace cpphf {

constexpr int kRtrMaxBlocks = 1024;
constexpr double kOccClip = 1.0e-8;  // OCC_CLIP (types.hpp)

// reduction result slots
enum : int {
    kSumDD = 0, kSumVD, kSumVV,              // direction pass: <d,d>, <v,d>, <v,v> (joint metric)
    kSumB1, kSumB2, kSumB3, kSumB4,          // HVP pass: Re<dX,HX>, sum w dp Hp, sum w dp, sum w Hp
    kSumRR, kSumA1, kSumA2, kSumA3, kSumA4,  // update pass: <r,r>, Re<rX,zX>, sum w rp z, sum w z, sum w rp
    kSumGV, kSumVHX, kSumVHP, kSumVVX, kSumVVP,  // model pass
    kSumW,                                   // sum_k w2d
    kNumSums
};

// Device scalars of a Newton solve (state slots 0/1 = current/trial, swapped by index)
struct RtrScalars {
    double mu[2];      // chemical potential of each state slot
    double energy[2];  // free energy (+ deflation bias) of each state slot
    double pen[2];     // deflation curvature 2 sum_i phi'(d_i^2) of each state slot
    double phi;        // deflation bias of the last evaluation
    double efin;       // energy of the final density
    double sums[kNumSums];
    unsigned counter;
    unsigned pad;
    double part[8 * kRtrMaxBlocks];
};

__device__ __forceinline__ double occ_clip(double p) { return fmin(fmax(p, kOccClip), 1.0 - kOccClip); }

size_t solve_rtr_workspace_bytes(const cpphf_kernel* K, const cpphf_dm_config* cfg);
int solve_rtr(const cpphf_kernel* K, const cpphf_dm_config* cfg, const double2* P0, double n_e,
              cpphf_project_fn project, void* puser, double2* Q_out, double* p_out, double2* D_out, double2* F_out,
              double* hist_E, double* hist_G, cpphf_dm_result* res, void* ws, size_t wsb, cudaStream_t st);

// Tiled kernels for nb in {2, 4, 6, 8} (rtr_small.cu); same contracts as the
// team kernels of rtr.cu.  Direction modes: 0 d = z(r), 1 d = z(r) + beta d,
// 2 d given, 3 as 1 with beta and shift_z formed on the device from the update
// pass's sums and rz_old.
bool rtr_small_supported(int nb);
int rtr_small_direction(const double2* rX, const double* rp, const double* eps, const double* p, const double* w,
                        const double2* Q, const double2* vX, const double* vp, double2* dX, double* dp, double2* dP,
                        int64_t nk, int nb, double T_r, double lam, double beta, double shift_z, double rz_old,
                        int mode, RtrScalars* R, cudaStream_t st);
int rtr_small_hvp(const double2* X, const double* dp, const double2* Q, const double* p, const double2* Ft,
                  const double2* Fr, const double2* h, const double2* dP, const double* pen, const double* w,
                  double2* HX, double* Hp, int64_t nk, int nb, double T_r, RtrScalars* R, cudaStream_t st);
int rtr_small_retract(const double2* D, const double2* Q, const double2* Ft, double2* Qt, double* ew, int64_t nk,
                      int nb, cudaStream_t st);

}  // namespace cpphf
