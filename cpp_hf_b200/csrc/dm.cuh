// Internal interface of the direct-minimisation per-k kernels.
#pragma once

#include "common.cuh"

namespace cpphf {

constexpr int kDmMaxPartials = 1024;

// Device-resident scalars of one DM iteration (written by last-block
// reductions, read by later kernels of the same iteration).
struct DmScalars {
    double mu;         // current chemical potential
    double mu_new;     // result of the in-loop mu solve
    double energy;     // E of the current iteration
    double grad_norm;
    double lam_pc;
    double beta;
    double tau0, tau_cur, tau_final;
    double omega0;
    int accepted;
    unsigned counter;  // last-block reduction counter (self-resetting)
    int iter;          // iterations since the start or the precision switch (CG restart count)
    int slot;          // trial of its pass the accepted one was (0: ew holds it, 1: ew2)
    double pad[1];
    double part[3 * kDmMaxPartials];
};

// One element of the SCF linear mix D + mixing (P_new - D) (solver_scf.hpp:395-401),
// shared by the mix kernel and the residual pass that fuses it, so both round alike;
// the Hermitian part of the mix m is then (m_ij + conj m_ji) / 2 per element.
__device__ __forceinline__ double2 scf_mix_elem(double2 d, double2 pn, double mixing) {
    return cadd(d, cscale(csub(pn, d), mixing));
}
__device__ __forceinline__ double2 scf_mix_herm(double2 mij, double2 mji) {
    return mk(0.5 * (mij.x + mji.x), 0.5 * (mij.y - mji.y));
}

int dm_check_nb(int64_t nb);
int dm_density(const double2* Q, const double* p, double2* P, int64_t nk, int nb, cudaStream_t st);
int dm_rotate(const double2* U, const double2* M, double2* Out, double* eps, int64_t nk, int nb, cudaStream_t st);
int dm_q_times_u(double2* Q, const double2* U, int64_t nk, int nb, cudaStream_t st);
int dm_occupations(const double* eps, const double* mu, double T_r, double* p, int64_t n, cudaStream_t st);
int dm_gradient(const double2* Ft, const double* p, const double* eps, const double* w, double2* G, double* g_p,
                int64_t nk, int nb, double T_r, double denom_scale, DmScalars* S, cudaStream_t st);
int dm_pr_beta(const double2* G, const double2* Gp, const double* g_p, const double* g_pp, const double* eps,
               const double* p, const double* w, int64_t nk, int nb, double T_r, int restart,
               DmScalars* S, cudaStream_t st);
int dm_direction(const double2* G, const double2* dQp, const double* g_p, const double* dpp, const double* eps,
                 const double* p, const double* w, double2* dQ, double* d_p, int64_t nk, int nb, double T_r,
                 double max_step, DmScalars* S, cudaStream_t st);
int dm_trial(const double2* V, const double2* Fe, const double* lam, const double* p, const double* d_p,
             const double* w, int64_t nk, int nb, double T_r, double shrink, int last_trial, double fallback,
             DmScalars* S, cudaStream_t st);
int dm_trial_lu(const double2* dQ, const double2* Ft, const double* p, const double* d_p, const double* w, int64_t nk,
                int nb, double T_r, double shrink, int last_trial, double fallback, DmScalars* S, cudaStream_t st);
int dm_retract_lu(double2* Q, const double2* dQ, const double2* Ft, double* ew, int64_t nk, int nb, const DmScalars* S,
                  cudaStream_t st);
int dm_retract(double2* Q, const double2* V, const double2* Fe, const double* lam, double* ew, int64_t nk, int nb,
               const DmScalars* S, cudaStream_t st);

}  // namespace cpphf
