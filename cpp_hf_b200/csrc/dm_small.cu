// Direct-minimisation per-k kernels specialised for small band counts
// (nb in {2, 4, 6, 8}; cpp_hf solver_dm.hpp:117-344).
//
// Tile kernels (density, rotation + gradient, Cayley trial, retraction): a
// group of GS = (nb rounded up to a power of two) threads owns one k-point and
// thread r owns row r of every matrix.  A CTA processes KT = 128/GS k-points
// per tile: whole k-blocks are staged through shared memory with coalesced,
// fully unrolled loads and stores into a padded layout (row stride nb + 1,
// matrix stride MS chosen so that a warp's row reads and the groups' broadcast
// reads fall in distinct banks).  Groups live inside one warp, so group-level
// ordering uses __syncwarp().
//
// Element kernels (PR+ beta, direction): one thread per matrix element, so
// every field access is coalesced; the per-row occupation terms run in a
// second loop, one row per thread (no divergent branch in the element loop).
#include "common.cuh"
#include "dm.cuh"
#include "dm_small.cuh"
#include "small_tile.cuh"
#include "team.cuh"

#include <algorithm>
#include <mutex>

namespace cpphf {

namespace {

using namespace tile;

constexpr double TINY_REAL = 1.0e-30;  // types.hpp:13
constexpr double LOGIT_CLIP = 1.0e-6;  // types.hpp:14
constexpr double OCC_CLIP = 1.0e-8;    // types.hpp:16

__device__ __forceinline__ double expit(double x) {
    if (x >= 0.0) return 1.0 / (1.0 + exp(-x));
    const double e = exp(x);
    return e / (1.0 + e);
}

// ---------------------------------------------------------------------------
// P = herm(Q diag(p) Q^H) with p = expit((mu - ew) / T_r) computed here
// (solver_dm.hpp:117-128 + 456-457/598-599); p written out.
// ---------------------------------------------------------------------------
// FROM_EW = false: the occupations are given in p (read, not written).
// The Q tiles come through two shared-memory stages filled by cp.async (the
// next tile's copies in flight while the current one is processed).
// Dynamic shared memory: sQ stage 0 | sQ stage 1, TILE double2 each; the
// product X = Q diag(p) Q^H of a tile replaces its Q stage once every row of Q
// has been read.
template <int NB, bool FROM_EW>
__global__ void __launch_bounds__(kThreads) k_dens_occ(const double2* __restrict__ Q, const double* __restrict__ ew,
                                                       const double* __restrict__ mu, double T_r, double* __restrict__ p,
                                                       double2* __restrict__ P, int64_t nk) {
    using G = Geo<NB>;
    extern __shared__ __align__(16) double2 dyn[];
    __shared__ double sp[G::KT * NB];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const double m = FROM_EW ? *mu : 0.0;
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    auto issue = [&](int64_t t, int s) {
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        tile_load_async<NB>(dyn + s * G::TILE, Q + (size_t)k0 * G::NB2, nkt);
    };
    if ((int64_t)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    cp_async_commit();
    int it = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int s = it & 1;
        if (t + (int64_t)gridDim.x < ntiles) issue(t + gridDim.x, s ^ 1);  // stage s ^ 1 was freed last iteration
        cp_async_commit();
        double2* sQ = dyn + s * G::TILE;
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        for (int e = threadIdx.x; e < nkt * NB; e += blockDim.x) {
            if (FROM_EW) {
                const double pv = expit((m - ew[k0 * NB + e]) / T_r);
                sp[e] = pv;
                p[k0 * NB + e] = pv;
            } else {
                sp[e] = p[k0 * NB + e];
            }
        }
        cp_async_wait_prev();
        __syncthreads();
        const bool live = grp < nkt && r < NB;
        double2 xr[NB];
        if (live) {
            const double2* q = sQ + grp * G::MS;
            const double* pk = sp + grp * NB;
            double2 qr[NB];
#pragma unroll
            for (int l = 0; l < NB; ++l) qr[l] = cscale(q[r * G::LD + l], pk[l]);
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                double2 acc = mk(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NB; ++l) cfmac(acc, qr[l], q[j * G::LD + l]);
                xr[j] = acc;
            }
        }
        __syncthreads();  // every row of Q is read: X takes the stage's place
        double2* sX = sQ;
        if (live) {
#pragma unroll
            for (int j = 0; j < NB; ++j) sX[grp * G::MS + r * G::LD + j] = xr[j];
        }
        __syncthreads();
        const int n = nkt * G::NB2;
#pragma unroll
        for (int u = 0; u < G::PER; ++u) {
            const int e = threadIdx.x + u * kThreads;
            if (e < n) {
                const int kl = e / G::NB2, rr = e - kl * G::NB2, i = rr / NB, j = rr - i * NB;
                const double2 a = sX[kl * G::MS + i * G::LD + j], b = sX[kl * G::MS + j * G::LD + i];
                P[(size_t)k0 * G::NB2 + e] = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Ft = Q^H F Q, eps = Re diag Ft, G = orbital gradient, g_p, and the
// reductions grad_norm, lam_pc (solver_dm.hpp:130-160, 497-519).
// Ft overwrites F.
// ---------------------------------------------------------------------------
// Two shared-memory stages of (Q, F) tiles: the next tile's asynchronous
// copies are in flight while the current one is processed.  Thread r forms
// column r of T = F Q and then column r of Ft = Q^H T from registers (the same
// products and summation order as row by row), so T never goes through shared
// memory; Ft's column replaces F's in the stage for the transposed reads of the
// gradient, and Ft and G go from registers straight to global memory (a
// group's eight columns of one row are one 128-byte run).
// Dynamic shared memory: stage s = { sQ, sT } at dyn + 2 s TILE.
template <int NB>
__global__ void __launch_bounds__(kThreads) k_rot_grad(const double2* __restrict__ Q, double2* F,
                                                       const double* __restrict__ p, const double* __restrict__ w,
                                                       double* __restrict__ eps, double2* __restrict__ Gout,
                                                       double* __restrict__ g_p, int64_t nk, double T_r,
                                                       double denom_scale, DmScalars* S) {
    using G = Geo<NB>;
    extern __shared__ __align__(16) double2 dyn[];
    __shared__ double red[64];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const double mu = S->mu;
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    double v[2] = {0.0, 0.0};
    auto issue = [&](int64_t t, int s) {
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        tile_load_async<NB>(dyn + 2 * s * G::TILE, Q + (size_t)k0 * G::NB2, nkt);
        tile_load_async<NB>(dyn + (2 * s + 1) * G::TILE, F + (size_t)k0 * G::NB2, nkt);
    };
    if ((int64_t)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    cp_async_commit();
    int it = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int s = it & 1;
        if (t + (int64_t)gridDim.x < ntiles) issue(t + gridDim.x, s ^ 1);  // stage s ^ 1 was freed last iteration
        cp_async_commit();
        cp_async_wait_prev();
        const double2* sQ = dyn + 2 * s * G::TILE;  // Q
        double2* sT = dyn + (2 * s + 1) * G::TILE;  // F, then Ft by columns
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        __syncthreads();
        const bool live = grp < nkt && r < NB;
        const int64_t k = k0 + grp;
        double2* tt = sT + grp * G::MS;
        const double2* q = sQ + grp * G::MS;
        const int rr = r < NB ? r : 0;
        double2 ftc[NB];  // column rr of Ft
        if (grp < nkt) {
            double2 tc[NB];  // column rr of T = F Q: T_ir = sum_l F_il Q_lr
            {
                double2 qc[NB];
#pragma unroll
                for (int l = 0; l < NB; ++l) qc[l] = q[l * G::LD + rr];
#pragma unroll
                for (int i = 0; i < NB; ++i) {
                    double2 acc = mk(0.0, 0.0);
#pragma unroll
                    for (int l = 0; l < NB; ++l) cfma(acc, tt[i * G::LD + l], qc[l]);
                    tc[i] = acc;
                }
            }
#pragma unroll
            for (int j = 0; j < NB; ++j) {  // Ft_jr = sum_i conj(Q_ij) T_ir
                double2 acc = mk(0.0, 0.0);
#pragma unroll
                for (int i = 0; i < NB; ++i) cfma(acc, cconj(q[i * G::LD + j]), tc[i]);
                ftc[j] = acc;
            }
        }
        __syncthreads();  // every read of F is done: Ft's columns take its place
        if (live) {
#pragma unroll
            for (int j = 0; j < NB; ++j) tt[j * G::LD + r] = ftc[j];
        }
        __syncthreads();
        if (live) {
            const double pr = p[k * NB + r];
            double er = ftc[0].x;
#pragma unroll
            for (int j = 1; j < NB; ++j)
                if (j == r) er = ftc[j].x;
            eps[k * NB + r] = er;
            double2* gf = F + (size_t)k * G::NB2 + r;     // column r of Ft over F
            double2* gg = Gout + (size_t)k * G::NB2 + r;  // column r of G
            double gsq = 0.0;
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                // g_jr = [(p_r - p_j) Ft_jr - conj((p_j - p_r) Ft_rj)] / 2, the
                // transpose partner of row r's element (its modulus is the same)
                double2 gv = mk(0.0, 0.0);
                if (j != r) {
                    const double pj = p[k * NB + j];
                    const double2 aij = cscale(ftc[j], pr - pj);
                    const double2 aji = cscale(tt[r * G::LD + j], pj - pr);
                    gv = mk(0.5 * (aij.x - aji.x), 0.5 * (aij.y + aji.y));
                }
                gf[j * NB] = ftc[j];
                gg[j * NB] = gv;
                gsq += gv.x * gv.x + gv.y * gv.y;
            }
            v[0] += w[k] * gsq;
            const double pv = fmin(fmax(pr, LOGIT_CLIP), 1.0 - LOGIT_CLIP);
            g_p[k * NB + r] = er + T_r * (log(pv) - log1p(-pv)) - mu;
            v[1] += er * er;
        }
        __syncthreads();  // the stage is free for the copies issued next iteration
    }
    double out[2];
    if (reduce_last_block<2>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        S->grad_norm = sqrt(fmax(0.0, out[0]));
        const double nv = (double)(nk * NB);
        const double scale = sqrt(out[1] / (nv > 1.0 ? nv : 1.0) + TINY_REAL);
        S->lam_pc = fmax(T_r, denom_scale * scale);
    }
}

// Two consecutive backtracking trials (solver_dm.hpp:577-589) per pass, by
// elimination: tau_a = tau_cur and tau_b = tau_a * shrink share the loads of d
// and Ft and run their eliminations in lockstep.  The last block then takes
// the reference's sequential decisions (accept tau_a on a strict decrease of
// the frozen free energy, else try tau_b, else shrink on), so the result is
// that of one pass per trial.  diag(U^H Ft U) goes to ew (tau_a) and ew2
// (tau_b), U(tau_a) to Ua and U(tau_b) to Ub; S->slot records which one the
// accepted trial left.  `bt` is the index of the pass's first trial; a pair
// past bt_max evaluates one trial.
// Dynamic shared memory: sD | sF, one d tile and one Ft tile, refilled by
// cp.async as soon as they are consumed: each thread copies its column of d
// into registers before the eliminations, so the next tile's d streams in
// during the eliminations and the diagonal, and the next Ft (needed only after
// the next tile's eliminations) streams in once the diagonal has read this
// one.  Each thread holds a column of U after the transposed eliminations and
// stores it directly: for a fixed row j the group's eight columns are one
// contiguous 128-byte run of U.
template <int NB>
__global__ void __launch_bounds__(kThreads, 3)
    k_trial2_small(const double2* __restrict__ dQ, const double2* __restrict__ Ft, const double* __restrict__ p,
                   const double* __restrict__ d_p, const double* __restrict__ w, double* __restrict__ ew,
                   double* __restrict__ ew2, double2* __restrict__ Ua, double2* __restrict__ Ub, int64_t nk,
                   double T_r, double shrink, int bt, int bt_max, double fallback, DmScalars* S) {
    if (S->accepted) return;  // grid-uniform
    using G = Geo<NB>;
    extern __shared__ __align__(16) double2 dyn[];
    double2* sD = dyn;
    double2* sF = dyn + G::TILE;
    __shared__ double2 sPiv[G::KT * 8 * NB];
    __shared__ double red[128];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const unsigned mask = group_mask<NB>(threadIdx.x & 31);
    const double tau_a = S->tau_cur;
    const double tau_b = tau_a * shrink;
    const bool two = bt + 1 < bt_max;  // grid-uniform
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    auto tile_k = [&](int64_t t) { return (int)((nk - t * G::KT) < G::KT ? (nk - t * G::KT) : G::KT); };
    if ((int64_t)blockIdx.x < ntiles) {
        tile_load_async<NB>(sD, dQ + (size_t)blockIdx.x * G::KT * G::NB2, tile_k(blockIdx.x));
        tile_load_async<NB>(sF, Ft + (size_t)blockIdx.x * G::KT * G::NB2, tile_k(blockIdx.x));
    }
    cp_async_commit();
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t k0 = t * G::KT;
        const int nkt = tile_k(t);
        const int64_t tn = t + gridDim.x;  // this block's next tile
        cp_async_wait_all();
        __syncthreads();  // this tile's d and Ft have landed
        const bool live = grp < nkt && r < NB;
        const int rr = r < NB ? r : 0;
        const int64_t k = k0 + grp;
        double2 dv[NB];  // column rr of d (transposed eliminations)
#pragma unroll
        for (int j = 0; j < NB; ++j) dv[j] = sD[grp * G::MS + j * G::LD + rr];
        __syncthreads();  // every column of d is in registers: the next d may land
        if (tn < ntiles) tile_load_async<NB>(sD, dQ + (size_t)tn * G::KT * G::NB2, tile_k(tn));
        cp_async_commit();
        double2 ua[NB], ub[NB];
        double da = 0.0, db = 0.0;
        if (grp < nkt) {
            // thread r: column r of U(tau_a) and U(tau_b)
            if (two) {
                row_cayley2_reg<NB>(dv, tau_a, tau_b, rr, sPiv + grp * 8 * NB, ua, ub, mask);
                col_diag_uhfu<NB, G::LD, true>(sF + grp * G::MS, ua, ub, da, db);
            } else {
                row_cayley_reg<NB>(dv, tau_a, rr, sPiv + grp * 8 * NB, ua, mask);
                col_diag_uhfu<NB, G::LD, false>(sF + grp * G::MS, ua, ub, da, db);
            }
        }
        __syncthreads();  // every read of Ft is done: the next Ft may land
        if (tn < ntiles) tile_load_async<NB>(sF, Ft + (size_t)tn * G::KT * G::NB2, tile_k(tn));
        cp_async_commit();
        if (live) {
            // both factors go out, so that the retraction reads the accepted one
            double2* ga = Ua + (size_t)k * G::NB2 + r;
#pragma unroll
            for (int j = 0; j < NB; ++j) ga[j * NB] = ua[j];
            if (two) {
                double2* gb = Ub + (size_t)k * G::NB2 + r;
#pragma unroll
                for (int j = 0; j < NB; ++j) gb[j * NB] = ub[j];
            }
            const double wk = w[k], pk = p[k * NB + r], dpk = d_p[k * NB + r];
            ew[k * NB + r] = da;
            const double pa = fmin(fmax(pk - tau_a * dpk, OCC_CLIP), 1.0 - OCC_CLIP);
            v[0] += wk * pa * da;
            v[1] -= wk * (pa * log(pa) + (1.0 - pa) * log1p(-pa));
            if (two) {
                ew2[k * NB + r] = db;
                const double pb = fmin(fmax(pk - tau_b * dpk, OCC_CLIP), 1.0 - OCC_CLIP);
                v[2] += wk * pb * db;
                v[3] -= wk * (pb * log(pb) + (1.0 - pb) * log1p(-pb));
            }
        }
    }
    cp_async_wait_all();
    double out[4];
    if (reduce_last_block<4>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        const double Tc = fmax(T_r, 1.0e-14);
        const double om_a = out[0] - Tc * out[1];
        if (om_a < S->omega0) {
            S->accepted = 1;
            S->tau_final = tau_a;
            S->slot = 0;
        } else {
            S->tau_cur = tau_a * shrink;
            if (bt == bt_max - 1) S->tau_final = S->tau0 * fallback;
            if (two) {
                const double om_b = out[2] - Tc * out[3];
                if (om_b < S->omega0) {
                    S->accepted = 1;
                    S->tau_final = tau_b;
                    S->slot = 1;
                } else {
                    S->tau_cur = tau_b * shrink;
                    if (bt + 1 == bt_max - 1) S->tau_final = S->tau0 * fallback;
                }
            }
        }
    }
}

// Retraction Q <- Q U(tau_final) and eps_work = diag(U^H Ft U).  After an
// accepted trial, U is the one its pass stored (Ua or Ub) and eps_work its
// diagonal (copied from ew2 when it was the second of its pass); for the
// fallback step both are computed here, U from d by elimination.
// Dynamic shared memory: four tiles (two (U, Q) stages for an accepted trial;
// d, Ft and Q for the fallback step).
template <int NB>
__global__ void __launch_bounds__(kThreads) k_retract_small(double2* Q, const double2* __restrict__ dQ,
                                                            const double2* __restrict__ Ft, double* __restrict__ ew,
                                                            const double* __restrict__ ew2,
                                                            const double2* __restrict__ Ua,
                                                            const double2* __restrict__ Ub, int64_t nk,
                                                            const DmScalars* S) {
    using G = Geo<NB>;
    extern __shared__ __align__(16) double2 dyn[];
    double2* sD = dyn;
    double2* sF = dyn + G::TILE;
    double2* sU = sD;  // U replaces d row by row once the elimination has read d
    double2* sQ = dyn + 2 * G::TILE;
    __shared__ double2 sPiv[G::KT * 4 * NB];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const unsigned mask = group_mask<NB>(threadIdx.x & 31);
    const double tau = S->tau_final;
    const bool need_diag = S->accepted == 0;                // grid-uniform: the fallback step
    const bool from_b = S->accepted != 0 && S->slot == 1;  // grid-uniform
    const double2* Uacc = from_b ? Ub : Ua;
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    if (!need_diag) {
        // accepted trial: Q <- Q U with U read back, two shared-memory stages of
        // (U, Q) tiles filled by cp.async (the next tile's copies in flight
        // while the current one is multiplied); thread r forms column r of Q U
        // (the same products in the same order as row by row) and stores it
        // directly (a group's eight columns of one row are one 128-byte run)
        auto issue = [&](int64_t t, int st) {
            const int64_t k0 = t * G::KT;
            const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
            tile_load_async<NB>(dyn + 2 * st * G::TILE, Uacc + (size_t)k0 * G::NB2, nkt);
            tile_load_async<NB>(dyn + (2 * st + 1) * G::TILE, Q + (size_t)k0 * G::NB2, nkt);
        };
        if ((int64_t)blockIdx.x < ntiles) issue(blockIdx.x, 0);
        cp_async_commit();
        int it = 0;
        for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
            const int st = it & 1;
            if (t + (int64_t)gridDim.x < ntiles) issue(t + gridDim.x, st ^ 1);  // freed last iteration
            cp_async_commit();
            cp_async_wait_prev();
            __syncthreads();
            const double2* su = dyn + 2 * st * G::TILE + grp * G::MS;
            const double2* sq = dyn + (2 * st + 1) * G::TILE + grp * G::MS;
            const int64_t k0 = t * G::KT;
            const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
            if (grp < nkt && r < NB) {
                const int64_t k = k0 + grp;
                if (from_b) ew[k * NB + r] = ew2[k * NB + r];
                double2 uc[NB];  // column r of U
#pragma unroll
                for (int l = 0; l < NB; ++l) uc[l] = su[l * G::LD + r];
                double2* gq = Q + (size_t)k * G::NB2 + r;
#pragma unroll
                for (int j = 0; j < NB; ++j) {  // (Q U)_jr
                    double2 acc = mk(0.0, 0.0);
#pragma unroll
                    for (int l = 0; l < NB; ++l) cfma(acc, sq[j * G::LD + l], uc[l]);
                    gq[j * NB] = acc;
                }
            }
            __syncthreads();  // the stage is free for the copies issued next iteration
        }
        return;
    }
    // fallback step: U(tau_final) by elimination and its eps_work
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        if (need_diag) {
            tile_load<NB>(sD, dQ + (size_t)k0 * G::NB2, nkt);
            tile_load<NB>(sF, Ft + (size_t)k0 * G::NB2, nkt);
        } else {
            tile_load<NB>(sU, Uacc + (size_t)k0 * G::NB2, nkt);
        }
        tile_load<NB>(sQ, Q + (size_t)k0 * G::NB2, nkt);
        __syncthreads();
        const bool live = grp < nkt && r < NB;
        const int rr = r < NB ? r : 0;
        const int64_t k = k0 + grp;
        if (need_diag && grp < nkt) {
            double2 u[NB];
            row_cayley<NB, G::LD>(sD + grp * G::MS, tau, rr, sPiv + grp * 4 * NB, u, mask);
            // (the elimination ends with a group barrier after its last read of d)
            if (live) {
#pragma unroll
                for (int j = 0; j < NB; ++j) sU[grp * G::MS + r * G::LD + j] = u[j];
            }
        }
        __syncwarp();
        if (grp < nkt) {
            if (need_diag) {
                double2 ftj[NB];
#pragma unroll
                for (int l = 0; l < NB; ++l) ftj[l] = sF[grp * G::MS + rr * G::LD + l];
                const double dr = row_diag_uhfu<NB, G::GS, G::LD>(ftj, sU + grp * G::MS, r, mask, live);
                if (live) ew[k * NB + r] = dr;
            } else if (from_b && live) {
                ew[k * NB + r] = ew2[k * NB + r];
            }
            if (live) {
                const double2* su = sU + grp * G::MS;
                double2* qrow = sQ + grp * G::MS + r * G::LD;
                double2 qr[NB];
#pragma unroll
                for (int l = 0; l < NB; ++l) qr[l] = qrow[l];
#pragma unroll
                for (int j = 0; j < NB; ++j) {
                    double2 acc = mk(0.0, 0.0);
#pragma unroll
                    for (int l = 0; l < NB; ++l) cfma(acc, qr[l], su[l * G::LD + j]);
                    qrow[j] = acc;  // only this thread reads or writes this row
                }
            }
        }
        __syncthreads();
        tile_store<NB>(Q + (size_t)k0 * G::NB2, sQ, nkt);
        __syncthreads();
    }
}

// Element kernels (PR+ beta, direction): a grid-stride loop over the matrix
// elements (coalesced), then one over the rows for the occupation terms.  At
// most 64 registers, so four 256-thread CTAs per SM keep their loads in
// flight (these kernels are bound by load latency).  The preconditioner
// 1 / sqrt(gap^2 + lambda^2) is one reciprocal square root per element.
constexpr int kThreadsE = 256;
constexpr int kUnrollE = 4;  // elements a thread has in flight in the element loops

// PR+ numerator / denominator -> beta (solver_dm.hpp:513-559)
template <int NB>
__global__ void __launch_bounds__(kThreadsE, 4) k_pr_beta_small(const double2* __restrict__ Gc, const double2* __restrict__ Gp,
                                                             const double* __restrict__ g_p,
                                                             const double* __restrict__ g_pp,
                                                             const double* __restrict__ eps,
                                                             const double* __restrict__ p, const double* __restrict__ w,
                                                             int64_t nk, double T_r, int restart, DmScalars* S) {
    __shared__ double red[96];
    const double lam = S->lam_pc, lam2 = lam * lam;
    double v[3] = {0.0, 0.0, 0.0};
    const int64_t nrow = nk * NB, nel = nrow * NB;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // matrix terms, one element per thread (coalesced): kUnrollE elements of a
    // thread have all their loads (G, G_prev, both eigenvalues, the weight)
    // issued before any is used, so a batch costs one memory latency
    struct Ld {
        double2 g, gp;
        double er, ej, wk;
    };
    auto load = [&](int64_t e) {
        const int64_t row = e / NB, k = row / NB;
        const int j = (int)(e - row * NB);
        return Ld{Gc[e], Gp[e], eps[row], eps[k * NB + j], w[k]};
    };
    auto term = [&](const Ld& x) {
        const double gap = x.er - x.ej;
        const double rb = rsqrt(gap * gap + lam2);
        const double2 d = mk(x.g.x * rb, x.g.y * rb);
        v[0] += x.wk * ((x.g.x * d.x + x.g.y * d.y) - (x.gp.x * d.x + x.gp.y * d.y));
        v[1] += x.wk * (x.gp.x * x.gp.x + x.gp.y * x.gp.y);
    };
    int64_t e = tid;
    for (; e + (kUnrollE - 1) * stride < nel; e += kUnrollE * stride) {
        Ld x[kUnrollE];
#pragma unroll
        for (int u = 0; u < kUnrollE; ++u) x[u] = load(e + u * stride);
#pragma unroll
        for (int u = 0; u < kUnrollE; ++u) term(x[u]);
    }
    for (; e < nel; e += stride) term(load(e));
    // occupation terms, one row per thread
    for (int64_t row = tid; row < nrow; row += stride) {
        const double wk = w[row / NB];
        const double ps = fmin(fmax(p[row], OCC_CLIP), 1.0 - OCC_CLIP);
        const double gr = g_p[row], gq = g_pp[row];
        const double h = gr / (T_r / (ps * (1.0 - ps)));
        v[2] += wk * (gr * h - gq * h);
        v[1] += wk * (gq * gq);
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

// direction + tau0 + Omega0 (solver_dm.hpp:556-573, 346-365)
template <int NB>
__global__ void __launch_bounds__(kThreadsE, 4) k_direction_small(const double2* __restrict__ Gc,
                                                               const double2* __restrict__ dQp,
                                                               const double* __restrict__ g_p,
                                                               const double* __restrict__ dpp,
                                                               const double* __restrict__ eps,
                                                               const double* __restrict__ p,
                                                               const double* __restrict__ w, double2* __restrict__ dQ,
                                                               double* __restrict__ d_p, int64_t nk, double T_r,
                                                               double max_step, DmScalars* S) {
    __shared__ double red[96];
    const double lam = S->lam_pc, lam2 = lam * lam, beta = S->beta;
    double v[3] = {0.0, 0.0, 0.0};
    const int64_t nrow = nk * NB, nel = nrow * NB;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // matrix terms, one element per thread (coalesced): kUnrollE elements of a
    // thread have all their loads (G, the previous direction, both
    // eigenvalues, the weight) issued before any is used
    const bool use_prev = beta != 0.0;
    struct Ld {
        double2 g, q;
        double er, ej, wk;
    };
    auto load = [&](int64_t e) {
        const int64_t row = e / NB, k = row / NB;
        const int j = (int)(e - row * NB);
        return Ld{Gc[e], use_prev ? dQp[e] : mk(0.0, 0.0), eps[row], eps[k * NB + j], w[k]};
    };
    auto term = [&](int64_t e, const Ld& x) {
        const double gap = x.er - x.ej;
        const double rb = rsqrt(gap * gap + lam2);
        const double2 d = mk(x.g.x * rb + beta * x.q.x, x.g.y * rb + beta * x.q.y);
        dQ[e] = d;
        v[0] += x.wk * (d.x * d.x + d.y * d.y);
    };
    int64_t e = tid;
    for (; e + (kUnrollE - 1) * stride < nel; e += kUnrollE * stride) {
        Ld x[kUnrollE];
#pragma unroll
        for (int u = 0; u < kUnrollE; ++u) x[u] = load(e + u * stride);
#pragma unroll
        for (int u = 0; u < kUnrollE; ++u) term(e + u * stride, x[u]);
    }
    for (; e < nel; e += stride) term(e, load(e));
    // occupation terms, one row per thread
    for (int64_t row = tid; row < nrow; row += stride) {
        const double wk = w[row / NB];
        const double ps = fmin(fmax(p[row], OCC_CLIP), 1.0 - OCC_CLIP);
        const double h = g_p[row] / (T_r / (ps * (1.0 - ps)));
        d_p[row] = h + beta * dpp[row];
        v[1] += wk * ps * eps[row];
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

// One resident wave of the element kernels (four 256-thread CTAs per SM), or
// fewer CTAs when the rows do not fill it.
unsigned rows_grid(int64_t nrow) {
    const int64_t want = (nrow + kThreadsE - 1) / kThreadsE;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, std::min<int64_t>(kDmMaxPartials, 4 * num_sms())));
}

// ---------------------------------------------------------------------------
// SCF residuals (solver_scf.hpp:64-75, 224-242): sum_k w_k |Pn - D|_F^2 and
// sum_k w_k |F D - D F|_F^2 into S->grad_norm and S->lam_pc; the commutator
// itself goes to comm_out when given (the C-DIIS residual).  With mix_out the
// pass also writes the linear mix herm(D + mixing (Pn - D)) (solver_scf.hpp:
// 395-401) from the tiles it holds; mix_out may be D (each tile is read into
// shared memory before it is written back).
// ---------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(kThreads, 3) k_scf_residuals_small(const double2* __restrict__ F, const double2* D,
                                                                  const double2* __restrict__ Pn,
                                                                  const double* __restrict__ w, int64_t nk,
                                                                  DmScalars* S, double2* __restrict__ comm_out,
                                                                  double2* mix_out, double mixing) {
    using G = Geo<NB>;
    extern __shared__ __align__(16) double2 dyn[];
    __shared__ double red[64];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    double v[2] = {0.0, 0.0};
    // two shared-memory stages of (F, D) tiles filled by cp.async: the next
    // tile's copies are in flight while the current one is reduced
    auto issue = [&](int64_t t, int st) {
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        tile_load_async<NB>(dyn + 2 * st * G::TILE, F + (size_t)k0 * G::NB2, nkt);
        tile_load_async<NB>(dyn + (2 * st + 1) * G::TILE, D + (size_t)k0 * G::NB2, nkt);
    };
    if ((int64_t)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    cp_async_commit();
    int it = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int st = it & 1;
        if (t + (int64_t)gridDim.x < ntiles) issue(t + gridDim.x, st ^ 1);  // freed last iteration
        cp_async_commit();
        double2* sF = dyn + 2 * st * G::TILE;
        const double2* sD = dyn + (2 * st + 1) * G::TILE;
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        const int n = nkt * G::NB2;
        double2 pv[G::PER];  // loaded while the stage's copies land
#pragma unroll
        for (int u = 0; u < G::PER; ++u) {
            const int e = threadIdx.x + u * kThreads;
            pv[u] = e < n ? Pn[(size_t)k0 * G::NB2 + e] : mk(0.0, 0.0);
        }
        cp_async_wait_prev();
        __syncthreads();
#pragma unroll
        for (int u = 0; u < G::PER; ++u) {
            const int e = threadIdx.x + u * kThreads;
            if (e < n) {
                const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
                const double2 d = csub(pv[u], sD[kl * G::MS + i * G::LD + j]);
                v[0] += w[k0 + kl] * (d.x * d.x + d.y * d.y);
            }
        }
        const bool live = grp < nkt && r < NB;
        double2 c[NB];
        if (live) {
            const double2* f = sF + grp * G::MS;
            const double2* dd = sD + grp * G::MS;
            double sc = 0.0;
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                double2 fp = mk(0.0, 0.0), pf = mk(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NB; ++l) {
                    cfma(fp, f[r * G::LD + l], dd[l * G::LD + j]);
                    cfma(pf, dd[r * G::LD + l], f[l * G::LD + j]);
                }
                c[j] = csub(fp, pf);
                sc += c[j].x * c[j].x + c[j].y * c[j].y;
            }
            v[1] += w[k0 + grp] * sc;
        }
        if (comm_out) {  // grid-uniform
            __syncthreads();  // every read of F is done
            if (live) {
#pragma unroll
                for (int j = 0; j < NB; ++j) sF[grp * G::MS + r * G::LD + j] = c[j];
            }
            __syncthreads();
            tile_store<NB>(comm_out + (size_t)k0 * G::NB2, sF, nkt);
        }
        if (mix_out) {  // grid-uniform
            __syncthreads();  // every read of F (or of the commutator tile) is done
            double2* sM = sF;  // the elementwise mix m = D + mixing (Pn - D)
#pragma unroll
            for (int u = 0; u < G::PER; ++u) {
                const int e = threadIdx.x + u * kThreads;
                if (e < n) {
                    const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
                    const int o = kl * G::MS + i * G::LD + j;
                    sM[o] = scf_mix_elem(sD[o], pv[u], mixing);
                }
            }
            __syncthreads();
            double2* sH = dyn + (2 * st + 1) * G::TILE;  // D's stage takes the Hermitian part
#pragma unroll
            for (int u = 0; u < G::PER; ++u) {
                const int e = threadIdx.x + u * kThreads;
                if (e < n) {
                    const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
                    sH[kl * G::MS + i * G::LD + j] =
                        scf_mix_herm(sM[kl * G::MS + i * G::LD + j], sM[kl * G::MS + j * G::LD + i]);
                }
            }
            __syncthreads();
            tile_store<NB>(mix_out + (size_t)k0 * G::NB2, sH, nkt);
        }
        __syncthreads();
    }
    double out[2];
    if (reduce_last_block<2>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        S->grad_norm = out[0];  // density residual^2 * weight_sum
        S->lam_pc = out[1];     // commutator residual^2 * weight_sum
    }
}

template <int NB>
constexpr size_t kDensSmem = 2 * sizeof(double2) * Geo<NB>::TILE;  // two Q stages (X replaces its Q)

template <int NB>
void small_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        raise_smem(k_trial2_small<NB>);
        raise_smem(k_rot_grad<NB>);
        raise_smem(k_dens_occ<NB, true>);
        raise_smem(k_dens_occ<NB, false>);
        raise_smem(k_retract_small<NB>);
        raise_smem(k_scf_residuals_small<NB>);
    });
}

// CTAs of a persistent tile kernel resident on the device at once (at most
// kDmMaxPartials, the size of the reduction partials)
template <class K>
int resident_ctas(K kern, size_t smem) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kThreads, smem);
    (void)cudaGetLastError();
    return std::max(1, std::min(kDmMaxPartials, std::max(per, 1) * num_sms()));
}

}  // namespace

bool dm_small_supported(int nb) { return nb == 2 || nb == 4 || nb == 6 || nb == 8; }

int dm_small_dens_occ(const double2* Q, const double* ew, const double* mu, double T_r, double* p, double2* P,
                      int64_t nk, int nb, cudaStream_t st) {
#define X(N)                                                                                                     \
    small_attrs<N>();                                                                                            \
    k_dens_occ<N, true><<<tiles_grid(nk, Geo<N>::KT, resident_ctas(k_dens_occ<N, true>, kDensSmem<N>)), kThreads,  \
                          kDensSmem<N>, st>>>(Q, ew, mu, T_r, p, P, nk);                                        \
    CPPHF_LAUNCH_CHECK("dens_occ");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int dm_small_density(const double2* Q, const double* p, double2* P, int64_t nk, int nb, cudaStream_t st) {
#define X(N)                                                                                                        \
    small_attrs<N>();                                                                                               \
    k_dens_occ<N, false><<<tiles_grid(nk, Geo<N>::KT, resident_ctas(k_dens_occ<N, false>, kDensSmem<N>)), kThreads, \
                           kDensSmem<N>, st>>>(                                                                      \
        Q, nullptr, nullptr, 1.0, const_cast<double*>(p), P, nk);                                                   \
    CPPHF_LAUNCH_CHECK("density");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int scf_small_residuals(const double2* F, const double2* D, const double2* Pn, const double* w, int64_t nk, int nb,
                        DmScalars* S, double2* comm_out, double2* mix_out, double mixing, cudaStream_t st) {
#define X(N)                                                                                                      \
    small_attrs<N>();                                                                                              \
    k_scf_residuals_small<N><<<tiles_grid(nk, Geo<N>::KT, resident_ctas(k_scf_residuals_small<N>, 4 * sizeof(double2) * Geo<N>::TILE)), \
                               kThreads, 4 * sizeof(double2) * Geo<N>::TILE, st>>>(F, D, Pn, w, nk, S,          \
                                                                                             comm_out, mix_out,    \
                                                                                             mixing);              \
    CPPHF_LAUNCH_CHECK("scf residuals");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int dm_small_rot_grad(const double2* Q, double2* F, const double* p, const double* w, double* eps, double2* Gout,
                      double* g_p, int64_t nk, int nb, double T_r, double denom_scale, DmScalars* S, cudaStream_t st) {
#define X(N)                                                                                                    \
    small_attrs<N>();                                                                                           \
    k_rot_grad<N><<<tiles_grid(nk, Geo<N>::KT, resident_ctas(k_rot_grad<N>, 4 * sizeof(double2) * Geo<N>::TILE)),   \
                    kThreads, 4 * sizeof(double2) * Geo<N>::TILE, st>>>(Q, F, p, w, eps, Gout, g_p, nk,        \
                                                                                   T_r, denom_scale, S);        \
    CPPHF_LAUNCH_CHECK("rot_grad");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int dm_small_pr_beta(const double2* Gc, const double2* Gp, const double* g_p, const double* g_pp, const double* eps,
                     const double* p, const double* w, int64_t nk, int nb, double T_r, int restart, DmScalars* S,
                     cudaStream_t st) {
#define X(N)                                                                                                     \
    k_pr_beta_small<N><<<rows_grid(nk * N), kThreadsE, 0, st>>>(Gc, Gp, g_p, g_pp, eps, p, w, nk, T_r, restart, \
                                                                    S);                                          \
    CPPHF_LAUNCH_CHECK("pr_beta");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int dm_small_direction(const double2* Gc, const double2* dQp, const double* g_p, const double* dpp, const double* eps,
                       const double* p, const double* w, double2* dQ, double* d_p, int64_t nk, int nb, double T_r,
                       double max_step, DmScalars* S, cudaStream_t st) {
#define X(N)                                                                                                        \
    k_direction_small<N><<<rows_grid(nk * N), kThreadsE, 0, st>>>(Gc, dQp, g_p, dpp, eps, p, w, dQ, d_p, nk, T_r, \
                                                                      max_step, S);                                 \
    CPPHF_LAUNCH_CHECK("direction");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int dm_small_trial2(const double2* dQ, const double2* Ft, const double* p, const double* d_p, const double* w,
                    double* ew, double* ew2, double2* Ua, double2* Ub, int64_t nk, int nb, double T_r, double shrink,
                    int bt, int bt_max, double fallback, DmScalars* S, cudaStream_t st) {
#define X(N)                                                                                                  \
    small_attrs<N>();                                                                                         \
    k_trial2_small<N><<<tiles_grid(nk, Geo<N>::KT,                                                            \
                                   std::min(3 * kDmMaxPartials / 4,                                           \
                                            (int)resident_ctas(k_trial2_small<N>, 2 * sizeof(double2) * Geo<N>::TILE))), \
                        kThreads, 2 * sizeof(double2) * Geo<N>::TILE, st>>>(dQ, Ft, p, d_p, w, ew, ew2, Ua, Ub, nk, \
                                                                           T_r, shrink, bt, bt_max, fallback, S); \
    CPPHF_LAUNCH_CHECK("trial pair");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int dm_small_retract(double2* Q, const double2* dQ, const double2* Ft, double* ew, const double* ew2,
                     const double2* Ua, const double2* Ub, int64_t nk, int nb, const DmScalars* S, cudaStream_t st) {
#define X(N)                                                                                                      \
    small_attrs<N>();                                                                                             \
    k_retract_small<N><<<tiles_grid(nk, Geo<N>::KT, resident_ctas(k_retract_small<N>, 4 * sizeof(double2) * Geo<N>::TILE)), \
                         kThreads, 4 * sizeof(double2) * Geo<N>::TILE, st>>>(Q, dQ, Ft, ew, ew2, Ua, Ub, nk, S);        \
    CPPHF_LAUNCH_CHECK("retract");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

}  // namespace cpphf
