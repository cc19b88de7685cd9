// Internal interface of the small-nb (2, 4, 6, 8) direct-minimisation kernels.
#pragma once

#include "common.cuh"
#include "dm.cuh"

namespace cpphf {

bool dm_small_supported(int nb);
// SCF density and commutator residuals (S->grad_norm, S->lam_pc), commutator to comm_out if given;
// with mix_out (which may be D itself) also the linear mix herm(D + mixing (Pn - D))
int scf_small_residuals(const double2* F, const double2* D, const double2* Pn, const double* w, int64_t nk, int nb,
                        DmScalars* S, double2* comm_out, double2* mix_out, double mixing, cudaStream_t st);
// P = herm(Q diag(p) Q^H) from given occupations p
int dm_small_density(const double2* Q, const double* p, double2* P, int64_t nk, int nb, cudaStream_t st);
int dm_small_dens_occ(const double2* Q, const double* ew, const double* mu, double T_r, double* p, double2* P,
                      int64_t nk, int nb, cudaStream_t st);
int dm_small_rot_grad(const double2* Q, double2* F, const double* p, const double* w, double* eps, double2* Gout,
                      double* g_p, int64_t nk, int nb, double T_r, double denom_scale, DmScalars* S, cudaStream_t st);
int dm_small_pr_beta(const double2* Gc, const double2* Gp, const double* g_p, const double* g_pp, const double* eps,
                     const double* p, const double* w, int64_t nk, int nb, double T_r, int restart,
                     DmScalars* S, cudaStream_t st);
int dm_small_direction(const double2* Gc, const double2* dQp, const double* g_p, const double* dpp, const double* eps,
                       const double* p, const double* w, double2* dQ, double* d_p, int64_t nk, int nb, double T_r,
                       double max_step, DmScalars* S, cudaStream_t st);
// Two consecutive line-search trials (bt, bt + 1 < bt_max) in one pass;
// diag(U^H Ft U) of the first to ew, of the second to ew2, the factors U to
// Ua and Ub (full fields).
int dm_small_trial2(const double2* dQ, const double2* Ft, const double* p, const double* d_p, const double* w,
                    double* ew, double* ew2, double2* Ua, double2* Ub, int64_t nk, int nb, double T_r, double shrink,
                    int bt, int bt_max, double fallback, DmScalars* S, cudaStream_t st);
// Q <- Q U(tau_final): U of the accepted trial read from Ua / Ub and its
// eps_work left in ew (taken from ew2 when that holds it); for the fallback
// step U (by elimination) and eps_work are computed here.
int dm_small_retract(double2* Q, const double2* dQ, const double2* Ft, double* ew, const double* ew2,
                     const double2* Ua, const double2* Ub, int64_t nk, int nb, const DmScalars* S, cudaStream_t st);

}  // namespace cpphf
