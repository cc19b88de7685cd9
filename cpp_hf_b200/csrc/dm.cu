// Per-k kernels of the direct-minimisation solver (cpp_hf solver_dm.hpp:117-388)
// and the spectral-Cayley C-ABI hooks.
//
// Dense per-k products run in teams (team.cuh).  Global scalars (gradient
// norm, preconditioner width, PR+ beta, step length, frozen free energies) are
// produced on the device by last-block-done reductions into a DmScalars
// record, so an iteration needs no host round trip except the convergence
// test.
#include "common.cuh"
#include "dm.cuh"
#include "dm_small.cuh"
#include "team.cuh"

#include <algorithm>
#include <mutex>

namespace cpphf {

namespace {

constexpr double TINY_REAL = 1.0e-30;  // types.hpp:13
constexpr double LOGIT_CLIP = 1.0e-6;  // types.hpp:14
constexpr double OCC_CLIP = 1.0e-8;    // types.hpp:16

__device__ __forceinline__ double expit(double x) {
    if (x >= 0.0) return 1.0 / (1.0 + exp(-x));
    const double e = exp(x);
    return e / (1.0 + e);
}

// ---------------------------------------------------------------------------
// density: P = herm(Q diag(p) Q^H)            (solver_dm.hpp:117-128 + herm)
// ---------------------------------------------------------------------------
template <bool WARP>
__global__ void k_density(const double2* __restrict__ Q, const double* __restrict__ p,
                          double2* __restrict__ P, int64_t nk, int nb) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    const int ld = nb + 1;
    double2* Qs = team_mats<WARP>(raw, nb, 2, nb, t.team);
    double2* Xs = Qs + team_mat_elems(nb);
    double* ps = reinterpret_cast<double*>(Xs + team_mat_elems(nb));
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Qs, Q + (size_t)k * nb * nb, nb, t);
        for (int i = t.tid; i < nb; i += t.nt) ps[i] = p[(size_t)k * nb + i];
        t.sync();
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            double2 acc = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) cfmac(acc, cscale(Qs[i * ld + l], ps[l]), Qs[j * ld + l]);
            Xs[i * ld + j] = acc;
        }
        t.sync();
        double2* Pk = P + (size_t)k * nb * nb;
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            const double2 a = Xs[i * ld + j], b = Xs[j * ld + i];
            Pk[e] = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        }
        t.sync();
    }
}

// ---------------------------------------------------------------------------
// rotate: Out = U^H M U per k; optional eps = Re diag(Out)   (solver_dm.hpp:130-139, 305-314)
// Out may alias M.
// ---------------------------------------------------------------------------
template <bool WARP>
__global__ void k_rotate(const double2* __restrict__ U, const double2* M, double2* Out,
                         double* __restrict__ eps, int64_t nk, int nb) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    const int ld = nb + 1;
    double2* Us = team_mats<WARP>(raw, nb, 3, 0, t.team);
    double2* Ms = Us + team_mat_elems(nb);
    double2* Ts = Ms + team_mat_elems(nb);
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Us, U + (size_t)k * nb * nb, nb, t);
        tload<WARP>(Ms, M + (size_t)k * nb * nb, nb, t);
        t.sync();
        tmm<false, false, WARP>(Ts, Ms, Us, nb, t);  // T = M U
        t.sync();
        tmm<true, false, WARP>(Ms, Us, Ts, nb, t);   // Out = U^H T
        t.sync();
        tstore<WARP>(Out + (size_t)k * nb * nb, Ms, nb, t);
        if (eps)
            for (int i = t.tid; i < nb; i += t.nt) eps[(size_t)k * nb + i] = Ms[i * ld + i].x;
        t.sync();
    }
}

// ---------------------------------------------------------------------------
// Cayley unitary U = V diag(c) V^H            (solver_dm.hpp:258-272)
// ---------------------------------------------------------------------------
template <bool WARP>
__global__ void k_cayley_unitary(const double2* __restrict__ V, const double* __restrict__ lam, double tau,
                                 double2* __restrict__ U, int64_t nk, int nb) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    const int ld = nb + 1;
    double2* Vs = team_mats<WARP>(raw, nb, 2, 0, t.team);
    double2* Cs = Vs + team_mat_elems(nb);
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Vs, V + (size_t)k * nb * nb, nb, t);
        t.sync();
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            Cs[i * ld + j] = cmul(Vs[i * ld + j], cayley_factor(lam[(size_t)k * nb + j], tau));
        }
        t.sync();
        double2* Uk = U + (size_t)k * nb * nb;
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            double2 acc = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) cfmac(acc, Cs[i * ld + l], Vs[j * ld + l]);
            Uk[e] = acc;
        }
        t.sync();
    }
}

// diag(U^H Ft U) from the spectrum: d_i = Re sum_j (V M)_ij conj(V_ij),
// M_ij = conj(c_i) Fe_ij c_j                   (solver_dm.hpp:277-303)
template <bool WARP>
__device__ __forceinline__ void team_diag_ufu(const double2* Vs, double2* Ms, double2* As, const double2* cs,
                                              double* out, int nb, const Team<WARP>& t) {
    const int ld = nb + 1;
    for (int e = t.tid; e < nb * nb; e += t.nt) {
        const int i = e / nb, j = e - i * nb;
        Ms[i * ld + j] = cmul(cmul(cconj(cs[i]), Ms[i * ld + j]), cs[j]);
    }
    t.sync();
    tmm<false, false, WARP>(As, Vs, Ms, nb, t);
    t.sync();
    for (int i = t.tid; i < nb; i += t.nt) {
        double s = 0.0;
        for (int j = 0; j < nb; ++j) {
            const double2 a = As[i * ld + j], v = Vs[i * ld + j];
            s += a.x * v.x + a.y * v.y;  // Re(a conj(v))
        }
        out[i] = s;
    }
}

template <bool WARP>
__global__ void k_diag_ufu(const double2* __restrict__ V, const double2* __restrict__ Fe,
                           const double* __restrict__ lam, double tau, double* __restrict__ diag,
                           int64_t nk, int nb) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    double2* Vs = team_mats<WARP>(raw, nb, 3, 2 * nb, t.team);
    double2* Ms = Vs + team_mat_elems(nb);
    double2* As = Ms + team_mat_elems(nb);
    double2* cs = As + team_mat_elems(nb);
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Vs, V + (size_t)k * nb * nb, nb, t);
        tload<WARP>(Ms, Fe + (size_t)k * nb * nb, nb, t);
        for (int i = t.tid; i < nb; i += t.nt) cs[i] = cayley_factor(lam[(size_t)k * nb + i], tau);
        t.sync();
        team_diag_ufu<WARP>(Vs, Ms, As, cs, diag + (size_t)k * nb, nb, t);
        t.sync();
    }
}

// ---------------------------------------------------------------------------
// gradient + g_p + reductions -> grad_norm, lam_pc   (solver_dm.hpp:142-160, 504-519)
// ---------------------------------------------------------------------------
__global__ void k_gradient(const double2* __restrict__ Ft, const double* __restrict__ p,
                           const double* __restrict__ eps, const double* __restrict__ w,
                           double2* __restrict__ G, double* __restrict__ g_p, int64_t nk, int nb,
                           double T_r, double denom_scale, DmScalars* S) {
    __shared__ double red[64];
    const int nb2 = nb * nb;
    const int64_t nel = nk * nb2;
    const double mu = S->mu;
    double v[2] = {0.0, 0.0};  // sum w |G|^2, sum eps^2
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / nb2;
        const int r = (int)(e - k * nb2);
        const int i = r / nb, j = r - i * nb;
        double2 g = mk(0.0, 0.0);
        if (i != j) {
            const double pi = p[k * nb + i], pj = p[k * nb + j];
            const double dij = pj - pi, dji = pi - pj;
            const double2 aij = cscale(Ft[(size_t)k * nb2 + i * nb + j], dij);
            const double2 aji = cscale(Ft[(size_t)k * nb2 + j * nb + i], dji);
            g = mk(0.5 * (aij.x - aji.x), 0.5 * (aij.y + aji.y));
        }
        G[e] = g;
        v[0] += w[k] * (g.x * g.x + g.y * g.y);
    }
    const int64_t nv = nk * nb;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nv; e += (int64_t)gridDim.x * blockDim.x) {
        const double pv = fmin(fmax(p[e], LOGIT_CLIP), 1.0 - LOGIT_CLIP);
        const double logit = log(pv) - log1p(-pv);
        g_p[e] = eps[e] + T_r * logit - mu;
        v[1] += eps[e] * eps[e];
    }
    double out[2];
    if (reduce_last_block<2>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        S->grad_norm = sqrt(fmax(0.0, out[0]));
        const double scale = sqrt(out[1] / (double)(nv > 1 ? nv : 1) + TINY_REAL);
        S->lam_pc = fmax(T_r, denom_scale * scale);
    }
}

// PR+ numerator / denominator -> beta                (solver_dm.hpp:513-559)
__global__ void k_pr_beta(const double2* __restrict__ G, const double2* __restrict__ Gp,
                          const double* __restrict__ g_p, const double* __restrict__ g_pp,
                          const double* __restrict__ eps, const double* __restrict__ p,
                          const double* __restrict__ w, int64_t nk, int nb, double T_r, int restart,
                          DmScalars* S) {
    __shared__ double red[96];
    const int nb2 = nb * nb;
    const int64_t nel = nk * nb2;
    const double lam = S->lam_pc;
    double v[3] = {0.0, 0.0, 0.0};  // ip(G,dQ) - ip(Gp,dQ), ip(Gp,Gp), vec parts
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / nb2;
        const int r = (int)(e - k * nb2);
        const int i = r / nb, j = r - i * nb;
        const double gap = eps[k * nb + i] - eps[k * nb + j];
        const double base = sqrt(gap * gap + lam * lam);
        const double2 g = G[e], gp = Gp[e];
        const double2 d = mk(g.x / base, g.y / base);
        const double wk = w[k];
        v[0] += wk * ((g.x * d.x + g.y * d.y) - (gp.x * d.x + gp.y * d.y));
        v[1] += wk * (gp.x * gp.x + gp.y * gp.y);
    }
    const int64_t nv = nk * nb;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nv; e += (int64_t)gridDim.x * blockDim.x) {
        const double ps = fmin(fmax(p[e], OCC_CLIP), 1.0 - OCC_CLIP);
        const double curv = T_r / (ps * (1.0 - ps));
        const double h = g_p[e] / curv;
        const double wk = w[e / nb];
        v[2] += wk * (g_p[e] * h - g_pp[e] * h);
        v[1] += wk * (g_pp[e] * g_pp[e]);
    }
    double out[3];
    if (reduce_last_block<3>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        const double num = out[0] + out[2];
        const double den = out[1];
        double beta = (den > TINY_REAL) ? fmax(0.0, num / den) : 0.0;
        beta = fmin(beta, 5.0);
        // the iteration count lives on the device (incremented here) so that an
        // iteration's launches do not depend on it
        const int iter = S->iter;
        if (iter == 0 || (restart > 0 && iter % restart == 0)) beta = 0.0;
        S->iter = iter + 1;
        S->beta = beta;
    }
}

// direction d = precond(G) + beta d_prev, d_p = h_p + beta d_p_prev; tau0, Omega0
// (solver_dm.hpp:556-573, 346-365)
__global__ void k_direction(const double2* __restrict__ G, const double2* __restrict__ dQp,
                            const double* __restrict__ g_p, const double* __restrict__ dpp,
                            const double* __restrict__ eps, const double* __restrict__ p,
                            const double* __restrict__ w, double2* __restrict__ dQ,
                            double* __restrict__ d_p, int64_t nk, int nb, double T_r, double max_step,
                            DmScalars* S) {
    __shared__ double red[96];
    const int nb2 = nb * nb;
    const int64_t nel = nk * nb2;
    const double lam = S->lam_pc, beta = S->beta;
    double v[3] = {0.0, 0.0, 0.0};  // ip(dQ,dQ), E0, S0
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / nb2;
        const int r = (int)(e - k * nb2);
        const int i = r / nb, j = r - i * nb;
        const double gap = eps[k * nb + i] - eps[k * nb + j];
        const double base = sqrt(gap * gap + lam * lam);
        const double2 g = G[e], q = dQp[e];
        const double2 d = mk(g.x / base + beta * q.x, g.y / base + beta * q.y);
        dQ[e] = d;
        v[0] += w[k] * (d.x * d.x + d.y * d.y);
    }
    const int64_t nv = nk * nb;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nv; e += (int64_t)gridDim.x * blockDim.x) {
        const double ps = fmin(fmax(p[e], OCC_CLIP), 1.0 - OCC_CLIP);
        const double curv = T_r / (ps * (1.0 - ps));
        const double h = g_p[e] / curv;
        d_p[e] = h + beta * dpp[e];
        const double wk = w[e / nb];
        v[1] += wk * ps * eps[e];
        v[2] -= wk * (ps * log(ps) + (1.0 - ps) * log1p(-ps));
    }
    double out[3];
    if (reduce_last_block<3>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        const double nrm = sqrt(fmax(0.0, out[0]));
        const double tau0 = fmin(1.0, max_step / fmax(nrm, TINY_REAL));
        S->tau0 = tau0;
        S->tau_cur = tau0;
        S->tau_final = tau0;
        S->accepted = 0;
        S->omega0 = out[1] - fmax(T_r, 1.0e-14) * out[2];
    }
}

// One backtracking trial: Omega(tau_cur) from diag_UFU and p - tau d_p.
// (solver_dm.hpp:577-589, 367-388)
template <bool WARP>
__global__ void k_trial(const double2* __restrict__ V, const double2* __restrict__ Fe,
                        const double* __restrict__ lam, const double* __restrict__ p,
                        const double* __restrict__ d_p, const double* __restrict__ w, int64_t nk, int nb,
                        double T_r, double shrink, int last_trial, double fallback, DmScalars* S) {
    if (S->accepted) return;  // grid-uniform
    extern __shared__ __align__(16) unsigned char raw[];
    __shared__ double red[64];
    Team<WARP> t;
    double2* Vs = team_mats<WARP>(raw, nb, 3, 3 * nb, t.team);
    double2* Ms = Vs + team_mat_elems(nb);
    double2* As = Ms + team_mat_elems(nb);
    double2* cs = As + team_mat_elems(nb);
    double* ds = reinterpret_cast<double*>(cs + nb);
    const double tau = S->tau_cur;
    double v[2] = {0.0, 0.0};
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Vs, V + (size_t)k * nb * nb, nb, t);
        tload<WARP>(Ms, Fe + (size_t)k * nb * nb, nb, t);
        for (int i = t.tid; i < nb; i += t.nt) cs[i] = cayley_factor(lam[(size_t)k * nb + i], tau);
        t.sync();
        team_diag_ufu<WARP>(Vs, Ms, As, cs, ds, nb, t);
        t.sync();
        const double wk = w[k];
        for (int i = t.tid; i < nb; i += t.nt) {
            const double pv = fmin(fmax(p[(size_t)k * nb + i] - tau * d_p[(size_t)k * nb + i], OCC_CLIP), 1.0 - OCC_CLIP);
            v[0] += wk * pv * ds[i];
            v[1] -= wk * (pv * log(pv) + (1.0 - pv) * log1p(-pv));
        }
        t.sync();
    }
    double out[2];
    if (reduce_last_block<2>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        const double om = out[0] - fmax(T_r, 1.0e-14) * out[1];
        if (om < S->omega0) {
            S->accepted = 1;
            S->tau_final = tau;
        } else {
            S->tau_cur = tau * shrink;
            if (last_trial) S->tau_final = S->tau0 * fallback;
        }
    }
}

// Retraction Q <- Q V diag(c) V^H and eps_work = diag_UFU(tau_final)
// (solver_dm.hpp:590-594, 328-344)
template <bool WARP>
__global__ void k_retract(double2* Q, const double2* __restrict__ V, const double2* __restrict__ Fe,
                          const double* __restrict__ lam, double* __restrict__ ew, int64_t nk, int nb,
                          const DmScalars* S, int use_tau_final) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    const int ld = nb + 1;
    double2* Vs = team_mats<WARP>(raw, nb, 3, 2 * nb, t.team);
    double2* Bs = Vs + team_mat_elems(nb);
    double2* Cs = Bs + team_mat_elems(nb);
    double2* cs = Cs + team_mat_elems(nb);
    const double tau = use_tau_final ? S->tau_final : 0.0;
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Vs, V + (size_t)k * nb * nb, nb, t);
        tload<WARP>(Bs, Q + (size_t)k * nb * nb, nb, t);
        for (int i = t.tid; i < nb; i += t.nt) cs[i] = cayley_factor(lam[(size_t)k * nb + i], tau);
        t.sync();
        tmm<false, false, WARP>(Cs, Bs, Vs, nb, t);  // C = Q V
        t.sync();
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            Cs[i * ld + j] = cmul(Cs[i * ld + j], cs[j]);
        }
        t.sync();
        tmm<false, true, WARP>(Bs, Cs, Vs, nb, t);  // Q_new = C V^H
        t.sync();
        tstore<WARP>(Q + (size_t)k * nb * nb, Bs, nb, t);
        tload<WARP>(Cs, Fe + (size_t)k * nb * nb, nb, t);
        t.sync();
        team_diag_ufu<WARP>(Vs, Cs, Bs, cs, ew + (size_t)k * nb, nb, t);
        t.sync();
    }
}


// ---------------------------------------------------------------------------
// Cayley unitary by elimination: U(tau) = (I + tau d / 2)^{-1} (I - tau d / 2).
// With H = i d Hermitian this equals V diag(c(tau, lam)) V^H of the spectral
// form (solver_dm.hpp:251-272), so every backtracking trial and the retraction
// need no eigendecomposition.  I + tau d / 2 has Hermitian part I (d is
// skew-Hermitian), so Gauss-Jordan elimination without pivoting is stable.
// On return Rs holds U (Ms is clobbered).
// ---------------------------------------------------------------------------
// d is read straight from the k-block in global memory (dense, row stride nb),
// so the team holds only M, the right-hand side R and one more matrix.
template <bool WARP>
__device__ __forceinline__ void team_cayley_lu(const double2* __restrict__ dk, double2* Ms, double2* Rs, double2* fs,
                                               double tau, int nb, const Team<WARP>& t) {
    const int ld = nb + 1;
    const double h = 0.5 * tau;
    for (int e = t.tid; e < nb * nb; e += t.nt) {
        const int i = e / nb, j = e - i * nb;
        const double2 a = cscale(dk[e], h);
        const double one = (i == j) ? 1.0 : 0.0;
        Ms[i * ld + j] = mk(one + a.x, a.y);
        Rs[i * ld + j] = mk(one - a.x, -a.y);
    }
    t.sync();
    for (int p = 0; p < nb; ++p) {
        const double2 piv = Ms[p * ld + p];
        const double inv = 1.0 / (piv.x * piv.x + piv.y * piv.y);
        for (int r = t.tid; r < nb; r += t.nt) {
            const double2 a = Ms[r * ld + p];
            fs[r] = (r == p) ? mk(0.0, 0.0) : cscale(cmulc(a, piv), inv);  // a / piv
        }
        t.sync();
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int r = e / nb, j = e - r * nb;
            if (r == p) continue;
            const double2 f = fs[r];
            Ms[r * ld + j] = csub(Ms[r * ld + j], cmul(f, Ms[p * ld + j]));
            Rs[r * ld + j] = csub(Rs[r * ld + j], cmul(f, Rs[p * ld + j]));
        }
        t.sync();
    }
    for (int e = t.tid; e < nb * nb; e += t.nt) {
        const int r = e / nb, j = e - r * nb;
        const double2 d = Ms[r * ld + r];
        const double inv = 1.0 / (d.x * d.x + d.y * d.y);
        Rs[r * ld + j] = cscale(cmulc(Rs[r * ld + j], d), inv);
    }
    t.sync();
}

// diag(U^H Ft U)_i = Re sum_j conj(U_ji) (Ft U)_ji ; Ws scratch
template <bool WARP>
__device__ __forceinline__ void team_diag_uhfu(const double2* Us, const double2* Fs, double2* Ws, double* out, int nb,
                                               const Team<WARP>& t) {
    const int ld = nb + 1;
    tmm<false, false, WARP>(Ws, Fs, Us, nb, t);
    t.sync();
    for (int i = t.tid; i < nb; i += t.nt) {
        double s = 0.0;
        for (int j = 0; j < nb; ++j) {
            const double2 u = Us[j * ld + i], w = Ws[j * ld + i];
            s += u.x * w.x + u.y * w.y;  // Re(conj(u) w)
        }
        out[i] = s;
    }
}

// One backtracking trial by elimination (solver_dm.hpp:577-589).
template <bool WARP>
__global__ void k_trial_lu(const double2* __restrict__ dQ, const double2* __restrict__ Ft,
                           const double* __restrict__ p, const double* __restrict__ d_p,
                           const double* __restrict__ w, int64_t nk, int nb, double T_r, double shrink,
                           int last_trial, double fallback, DmScalars* S) {
    if (S->accepted) return;  // grid-uniform
    extern __shared__ __align__(16) unsigned char raw[];
    __shared__ double red[64];
    Team<WARP> t;
    double2* Ms = team_mats<WARP>(raw, nb, 3, 3 * nb, t.team);
    double2* Rs = Ms + team_mat_elems(nb);
    double2* Fs = Rs + team_mat_elems(nb);
    double2* fs = Fs + team_mat_elems(nb);
    double* ds = reinterpret_cast<double*>(fs + nb);
    const double tau = S->tau_cur;
    double v[2] = {0.0, 0.0};
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Fs, Ft + (size_t)k * nb * nb, nb, t);
        team_cayley_lu<WARP>(dQ + (size_t)k * nb * nb, Ms, Rs, fs, tau, nb, t);
        team_diag_uhfu<WARP>(Rs, Fs, Ms, ds, nb, t);
        t.sync();
        const double wk = w[k];
        for (int i = t.tid; i < nb; i += t.nt) {
            const double pv = fmin(fmax(p[(size_t)k * nb + i] - tau * d_p[(size_t)k * nb + i], OCC_CLIP), 1.0 - OCC_CLIP);
            v[0] += wk * pv * ds[i];
            v[1] -= wk * (pv * log(pv) + (1.0 - pv) * log1p(-pv));
        }
        t.sync();
    }
    double out[2];
    if (reduce_last_block<2>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        const double om = out[0] - fmax(T_r, 1.0e-14) * out[1];
        if (om < S->omega0) {
            S->accepted = 1;
            S->tau_final = tau;
        } else {
            S->tau_cur = tau * shrink;
            if (last_trial) S->tau_final = S->tau0 * fallback;
        }
    }
}

// Retraction by elimination: Q <- Q U(tau_final), eps_work = diag(U^H Ft U).
template <bool WARP>
__global__ void k_retract_lu(double2* Q, const double2* __restrict__ dQ, const double2* __restrict__ Ft,
                             double* __restrict__ ew, int64_t nk, int nb, const DmScalars* S) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    double2* Ms = team_mats<WARP>(raw, nb, 3, 2 * nb, t.team);
    double2* Rs = Ms + team_mat_elems(nb);
    double2* Fs = Rs + team_mat_elems(nb);
    double2* fs = Fs + team_mat_elems(nb);
    const double tau = S->tau_final;
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Fs, Ft + (size_t)k * nb * nb, nb, t);
        team_cayley_lu<WARP>(dQ + (size_t)k * nb * nb, Ms, Rs, fs, tau, nb, t);
        team_diag_uhfu<WARP>(Rs, Fs, Ms, ew + (size_t)k * nb, nb, t);
        t.sync();
        tload<WARP>(Fs, Q + (size_t)k * nb * nb, nb, t);  // Ft is done: Q takes its place
        t.sync();
        tmm<false, false, WARP>(Ms, Fs, Rs, nb, t);  // Q U
        t.sync();
        tstore<WARP>(Q + (size_t)k * nb * nb, Ms, nb, t);
        t.sync();
    }
}

// p = expit((mu - eps) / T_r)  (solver_dm.hpp:456-457, 598-599)
__global__ void k_occupations(const double* __restrict__ eps, const double* __restrict__ mu, double T_r,
                              double* __restrict__ p, int64_t n) {
    const double m = *mu;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        p[e] = expit((m - eps[e]) / T_r);
}

// Q <- Q U (solver_dm.hpp:317-326)
template <bool WARP>
__global__ void k_q_times_u(double2* Q, const double2* __restrict__ U, int64_t nk, int nb) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    double2* As = team_mats<WARP>(raw, nb, 3, 0, t.team);
    double2* Bs = As + team_mat_elems(nb);
    double2* Cs = Bs + team_mat_elems(nb);
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(As, Q + (size_t)k * nb * nb, nb, t);
        tload<WARP>(Bs, U + (size_t)k * nb * nb, nb, t);
        t.sync();
        tmm<false, false, WARP>(Cs, As, Bs, nb, t);
        t.sync();
        tstore<WARP>(Q + (size_t)k * nb * nb, Cs, nb, t);
        t.sync();
    }
}

template <class Kfn>
void set_max_smem(Kfn f) {
    raise_smem(f);
}

void init_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        set_max_smem(k_density<true>);
        set_max_smem(k_density<false>);
        set_max_smem(k_rotate<true>);
        set_max_smem(k_rotate<false>);
        set_max_smem(k_cayley_unitary<true>);
        set_max_smem(k_cayley_unitary<false>);
        set_max_smem(k_diag_ufu<true>);
        set_max_smem(k_diag_ufu<false>);
        set_max_smem(k_trial<true>);
        set_max_smem(k_trial<false>);
        set_max_smem(k_retract<true>);
        set_max_smem(k_retract<false>);
        set_max_smem(k_q_times_u<true>);
        set_max_smem(k_q_times_u<false>);
        set_max_smem(k_trial_lu<true>);
        set_max_smem(k_trial_lu<false>);
        set_max_smem(k_retract_lu<true>);
        set_max_smem(k_retract_lu<false>);
    });
}

}  // namespace

int dm_check_nb(int64_t nb) {
    if (nb < 1) return fail(CPPHF_ERR_INVALID, "nb must be positive");
    // three team matrices of nb x (nb + 1) complex128 must fit in 227 KB (nb <= 68)
    if (sizeof(double2) * team_mat_elems((int)nb) * 3 + 64 * sizeof(double) + 4 * nb * sizeof(double2) > 227 * 1024)
        return fail(CPPHF_ERR_UNSUPPORTED, "nb too large for the per-k shared-memory kernels");
    return CPPHF_OK;
}

int dm_density(const double2* Q, const double* p, double2* P, int64_t nk, int nb, cudaStream_t st) {
    if (dm_small_supported(nb)) return dm_small_density(Q, p, P, nk, nb, st);
    init_attrs();
    const TeamLaunch L = team_launch(nk, nb);
    TEAM_DISPATCH(L, k_density, 2, nb, Q, p, P, nk, nb);
    return CPPHF_OK;
}

int dm_rotate(const double2* U, const double2* M, double2* Out, double* eps, int64_t nk, int nb, cudaStream_t st) {
    init_attrs();
    const TeamLaunch L = team_launch(nk, nb);
    TEAM_DISPATCH(L, k_rotate, 3, 0, U, M, Out, eps, nk, nb);
    return CPPHF_OK;
}

int dm_q_times_u(double2* Q, const double2* U, int64_t nk, int nb, cudaStream_t st) {
    init_attrs();
    const TeamLaunch L = team_launch(nk, nb);
    TEAM_DISPATCH(L, k_q_times_u, 3, 0, Q, U, nk, nb);
    return CPPHF_OK;
}

int dm_occupations(const double* eps, const double* mu, double T_r, double* p, int64_t n, cudaStream_t st) {
    k_occupations<<<flat_grid(n, 256), 256, 0, st>>>(eps, mu, T_r, p, n);
    CPPHF_LAUNCH_CHECK("occupations");
    return CPPHF_OK;
}

int dm_gradient(const double2* Ft, const double* p, const double* eps, const double* w, double2* G,
                double* g_p, int64_t nk, int nb, double T_r, double denom_scale, DmScalars* S, cudaStream_t st) {
    k_gradient<<<flat_grid(nk * nb * nb, 256), 256, 0, st>>>(Ft, p, eps, w, G, g_p, nk, nb, T_r, denom_scale, S);
    CPPHF_LAUNCH_CHECK("gradient");
    return CPPHF_OK;
}

int dm_pr_beta(const double2* G, const double2* Gp, const double* g_p, const double* g_pp, const double* eps,
               const double* p, const double* w, int64_t nk, int nb, double T_r, int restart, DmScalars* S,
               cudaStream_t st) {
    k_pr_beta<<<flat_grid(nk * nb * nb, 256), 256, 0, st>>>(G, Gp, g_p, g_pp, eps, p, w, nk, nb, T_r, restart, S);
    CPPHF_LAUNCH_CHECK("pr_beta");
    return CPPHF_OK;
}

int dm_direction(const double2* G, const double2* dQp, const double* g_p, const double* dpp, const double* eps,
                 const double* p, const double* w, double2* dQ, double* d_p, int64_t nk, int nb, double T_r,
                 double max_step, DmScalars* S, cudaStream_t st) {
    k_direction<<<flat_grid(nk * nb * nb, 256), 256, 0, st>>>(G, dQp, g_p, dpp, eps, p, w, dQ, d_p, nk, nb, T_r,
                                                              max_step, S);
    CPPHF_LAUNCH_CHECK("direction");
    return CPPHF_OK;
}

int dm_trial(const double2* V, const double2* Fe, const double* lam, const double* p, const double* d_p,
             const double* w, int64_t nk, int nb, double T_r, double shrink, int last_trial, double fallback,
             DmScalars* S, cudaStream_t st) {
    init_attrs();
    TeamLaunch L = team_launch(nk, nb);
    L.grid = std::min<unsigned>(L.grid, kDmMaxPartials);
    TEAM_DISPATCH(L, k_trial, 3, 3 * nb, V, Fe, lam, p, d_p, w, nk, nb, T_r, shrink, last_trial, fallback, S);
    return CPPHF_OK;
}

int dm_trial_lu(const double2* dQ, const double2* Ft, const double* p, const double* d_p, const double* w, int64_t nk,
                int nb, double T_r, double shrink, int last_trial, double fallback, DmScalars* S, cudaStream_t st) {
    init_attrs();
    TeamLaunch L = team_launch(nk, nb);
    L.grid = std::min<unsigned>(L.grid, kDmMaxPartials);
    TEAM_DISPATCH(L, k_trial_lu, 3, 3 * nb, dQ, Ft, p, d_p, w, nk, nb, T_r, shrink, last_trial, fallback, S);
    return CPPHF_OK;
}

int dm_retract_lu(double2* Q, const double2* dQ, const double2* Ft, double* ew, int64_t nk, int nb, const DmScalars* S,
                  cudaStream_t st) {
    init_attrs();
    const TeamLaunch L = team_launch(nk, nb);
    TEAM_DISPATCH(L, k_retract_lu, 3, 2 * nb, Q, dQ, Ft, ew, nk, nb, S);
    return CPPHF_OK;
}

int dm_retract(double2* Q, const double2* V, const double2* Fe, const double* lam, double* ew, int64_t nk, int nb,
               const DmScalars* S, cudaStream_t st) {
    init_attrs();
    const TeamLaunch L = team_launch(nk, nb);
    TEAM_DISPATCH(L, k_retract, 3, 2 * nb, Q, V, Fe, lam, ew, nk, nb, S, 1);
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

int cpphf_cayley_unitary(const void* V, const double* lam, double tau, void* U, int64_t batch, int64_t nb,
                         void* stream) {
    using namespace cpphf;
    CPPHF_TRY(dm_check_nb(nb));
    if (batch == 0) return CPPHF_OK;
    init_attrs();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const TeamLaunch L = team_launch(batch, (int)nb);
    const int nbi = (int)nb;
    {
        const int nb = nbi;
        TEAM_DISPATCH(L, k_cayley_unitary, 2, 0, static_cast<const double2*>(V), lam, tau,
                      static_cast<double2*>(U), batch, nb);
    }
    return CPPHF_OK;
}

int cpphf_diag_ufu(const void* V, const void* Ft_eig, const double* lam, double tau, double* diag, int64_t batch,
                   int64_t nb, void* stream) {
    using namespace cpphf;
    CPPHF_TRY(dm_check_nb(nb));
    if (batch == 0) return CPPHF_OK;
    init_attrs();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const TeamLaunch L = team_launch(batch, (int)nb);
    const int nbi = (int)nb;
    {
        const int nb = nbi;
        TEAM_DISPATCH(L, k_diag_ufu, 3, 2 * nb, static_cast<const double2*>(V),
                      static_cast<const double2*>(Ft_eig), lam, tau, diag, batch, nb);
    }
    return CPPHF_OK;
}

}  // extern "C"
