// Trust-region Newton per-k kernels for small band counts (nb in {2, 4, 6, 8};
// cpp_hf solver_rtr.hpp:55-111, 380-396).  Same tile scheme as the small-nb
// direct-minimisation kernels: a group of GS threads owns one k-point, thread r
// owns row r of every matrix, tiles of KT k-points are staged through shared
// memory with coalesced loads and stores, and every field load of a tile is
// issued before its first use.
#include "common.cuh"
#include "rtr.cuh"
#include "small_tile.cuh"
#include "team.cuh"

#include <mutex>

namespace cpphf {

namespace {

using namespace tile;

// ---------------------------------------------------------------------------
// Direction d (mode 0: z(r); 1: z(r) + beta d; 2: d given; 3: as 1 with beta
// and shift_z formed from the update pass's sums), one element per thread
// (coalesced), with the sums <d,d>, <v,d>, <v,v> in the joint metric.
// z(r) = rX / sqrt(gap^2 + lam^2) and rp p(1-p)/T - shift_z.
// ---------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(256, 4) k_rtr_dir_elem(const double2* __restrict__ rX, const double* __restrict__ rp,
                                                      const double* __restrict__ eps, const double* __restrict__ p,
                                                      const double* __restrict__ w, const double2* __restrict__ vX,
                                                      const double* __restrict__ vp, double2* dX, double* dp,
                                                      int64_t nk, double T_r, double lam, double beta, double shift_z,
                                                      double rz_old, int mode, RtrScalars* R) {
    __shared__ double red[32 * 3];
    if (mode == 3) {  // beta and shift_z from the preceding update pass (same arithmetic as the host)
        const double den = R->sums[kSumW] * (double)NB;
        shift_z = den > 0.0 ? R->sums[kSumA3] / den : 0.0;
        beta = (R->sums[kSumA1] + R->sums[kSumA2] - shift_z * R->sums[kSumA4]) / rz_old;
        mode = 1;
    }
    const double lam2 = lam * lam;
    const int64_t nrow = nk * NB, nel = nrow * NB;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double acc[3] = {0.0, 0.0, 0.0};
    // U elements per round, their loads issued before any is used (the pass is
    // bound by load latency); each thread still sums its elements in index order
    constexpr int U = 2;
    for (int64_t eb = tid; eb < nel; eb += U * stride) {
        double2 rv[U], ov[U], xv[U];
        double ea[U], ec[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t e = eb + u * stride;
            rv[u] = ov[u] = xv[u] = mk(0.0, 0.0);
            ea[u] = ec[u] = 0.0;
            if (e < nel) {
                if (mode == 2) {
                    ov[u] = dX[e];
                } else {
                    const int64_t row = e / NB, k = row / NB;
                    const int j = (int)(e - row * NB);
                    rv[u] = rX[e];
                    if (mode == 1) ov[u] = dX[e];
                    ea[u] = eps[row];
                    ec[u] = eps[k * NB + j];
                }
                if (vX) xv[u] = vX[e];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t e = eb + u * stride;
            if (e < nel) {
                double2 d;
                if (mode == 2) {
                    d = ov[u];
                } else {
                    const double gap = ea[u] - ec[u];
                    const double sc = sqrt(gap * gap + lam2);
                    d = mk(rv[u].x / sc, rv[u].y / sc);
                    if (mode == 1) d = mk(d.x + beta * ov[u].x, d.y + beta * ov[u].y);
                    dX[e] = d;
                }
                acc[0] += d.x * d.x + d.y * d.y;
                if (vX) {
                    acc[1] += xv[u].x * d.x + xv[u].y * d.y;
                    acc[2] += xv[u].x * xv[u].x + xv[u].y * xv[u].y;
                }
            }
        }
    }
    for (int64_t q = tid; q < nrow; q += stride) {
        double d;
        if (mode == 2) {
            d = dp[q];
        } else {
            const double pc = occ_clip(p[q]);
            const double z = rp[q] * pc * (1.0 - pc) / T_r - shift_z;
            d = mode == 0 ? z : z + beta * dp[q];
            dp[q] = d;
        }
        const double wk = w[q / NB];
        acc[0] += wk * d * d;
        if (vp) {
            const double v = vp[q];
            acc[1] += wk * v * d;
            acc[2] += wk * v * v;
        }
    }
    double out[3];
    if (reduce_last_block<3>(acc, R->part, &R->counter, out, red) && threadIdx.x == 0) {
        R->sums[kSumDD] = out[0];
        R->sums[kSumVD] = out[1];
        R->sums[kSumVV] = out[2];
    }
}

// ---------------------------------------------------------------------------
// Density variation of a direction: dP = herm(Q M Q^H) with M = [X, diag p]
// off the diagonal (X_ij (p_j - p_i)) and dp on it (solver_rtr.hpp:61-75).
// ---------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(kThreads) k_rtr_dP_small(const double2* __restrict__ Q,
                                                           const double2* __restrict__ X,
                                                           const double* __restrict__ dp,
                                                           const double* __restrict__ p, double2* __restrict__ dP,
                                                           int64_t nk) {
    using G = Geo<NB>;
    __shared__ double2 sQ[G::TILE];
    __shared__ double2 sM[G::TILE];
    __shared__ double sdp[G::KT * NB];
    __shared__ double sp[G::KT * NB];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const unsigned mask = group_mask<NB>(threadIdx.x & 31);
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        const int n = nkt * G::NB2;
        tile_load<NB>(sQ, Q + (size_t)k0 * G::NB2, nkt);
        tile_load<NB>(sM, X + (size_t)k0 * G::NB2, nkt);
        for (int e = threadIdx.x; e < nkt * NB; e += kThreads) {
            sdp[e] = dp[(size_t)k0 * NB + e];
            sp[e] = p[(size_t)k0 * NB + e];
        }
        __syncthreads();
        if (grp < nkt) {
            const int rr = r < NB ? r : 0;
            const double2* q = sQ + grp * G::MS;
            double2* m = sM + grp * G::MS;
            const double* pk = sp + grp * NB;
            const double* dk = sdp + grp * NB;
            double2 tr[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) {  // (Q M)_rj, M formed from X on the fly
                double2 a = mk(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NB; ++l) {
                    const double2 mlj = (l == j) ? mk(dk[l], 0.0) : cscale(m[l * G::LD + j], pk[j] - pk[l]);
                    cfma(a, q[rr * G::LD + l], mlj);
                }
                tr[j] = a;
            }
            double2 dr[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) {  // ((Q M) Q^H)_rj
                double2 a = mk(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NB; ++l) cfmac(a, tr[l], q[j * G::LD + l]);
                dr[j] = a;
            }
            __syncwarp(mask);  // every row of X has been read
            if (r < NB) {
#pragma unroll
                for (int j = 0; j < NB; ++j) m[rr * G::LD + j] = dr[j];
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < n; e += kThreads) {
            const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
            const double2 a = sM[kl * G::MS + i * G::LD + j], b = sM[kl * G::MS + j * G::LD + i];
            dP[(size_t)k0 * G::NB2 + e] = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Hessian-vector product assembly: R = F[dP] - h (+ pen dP), St = Q^H (R Q),
// A = (Ft X - X Ft) + St, HX = (C - C^H)/2 off the diagonal with
// C_ij = (dp_j - dp_i) Ft_ij + (p_j - p_i) A_ij, Hp = Re A_bb + T dp_b /
// (pc (1 - pc)) before the projection; sums Re<X,HX>, sum w dp Hp, sum w dp,
// sum w Hp.  Dynamic shared memory: sQ (Q, then X) | sR | sF; X is loaded once
// Q^H (R Q) is formed, so three tiles suffice (three CTAs per SM).
// ---------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(kThreads) k_rtr_hvp_small(
    const double2* __restrict__ X, const double* __restrict__ dp, const double2* __restrict__ Q,
    const double* __restrict__ p, const double2* __restrict__ Ft, const double2* __restrict__ Fr,
    const double2* __restrict__ h, const double2* __restrict__ dP, const double* __restrict__ pen,
    const double* __restrict__ w, double2* __restrict__ HX, double* __restrict__ Hp, int64_t nk, double T_r,
    RtrScalars* R) {
    using G = Geo<NB>;
    extern __shared__ __align__(16) double2 dyn[];
    double2* sQ = dyn;
    double2* sR = dyn + G::TILE;
    double2* sF = dyn + 2 * G::TILE;
    double2* sX = sQ;
    __shared__ double sdp[G::KT * NB];
    __shared__ double sp[G::KT * NB];
    __shared__ double red[32 * 4];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const unsigned mask = group_mask<NB>(threadIdx.x & 31);
    const double pc_ = pen ? *pen : 0.0;
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        const int n = nkt * G::NB2;
        tile_load<NB>(sQ, Q + (size_t)k0 * G::NB2, nkt);
        tile_load<NB>(sF, Ft + (size_t)k0 * G::NB2, nkt);
        {
            double2 fv[G::PER], hv[G::PER], pv[G::PER];
#pragma unroll
            for (int u = 0; u < G::PER; ++u) {
                const int e = threadIdx.x + u * kThreads;
                const size_t g = (size_t)k0 * G::NB2 + e;
                fv[u] = hv[u] = pv[u] = mk(0.0, 0.0);
                if (e < n) {
                    fv[u] = Fr[g];
                    hv[u] = h[g];
                    if (pc_ != 0.0) pv[u] = dP[g];
                }
            }
#pragma unroll
            for (int u = 0; u < G::PER; ++u) {
                const int e = threadIdx.x + u * kThreads;
                if (e < n) {
                    const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
                    double2 v = csub(fv[u], hv[u]);
                    if (pc_ != 0.0) v = mk(v.x + pc_ * pv[u].x, v.y + pc_ * pv[u].y);
                    sR[kl * G::MS + i * G::LD + j] = v;
                }
            }
        }
        for (int e = threadIdx.x; e < nkt * NB; e += kThreads) {
            sdp[e] = dp[(size_t)k0 * NB + e];
            sp[e] = p[(size_t)k0 * NB + e];
        }
        __syncthreads();
        double2 v[NB];
        if (grp < nkt) {
            const int rr = r < NB ? r : 0;
            const bool live = r < NB;
            const double2* q = sQ + grp * G::MS;
            double2* rm = sR + grp * G::MS;
#pragma unroll
            for (int j = 0; j < NB; ++j) {  // (R Q)_rj
                double2 a = mk(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NB; ++l) cfma(a, rm[rr * G::LD + l], q[l * G::LD + j]);
                v[j] = a;
            }
            __syncwarp(mask);
            if (live) {
#pragma unroll
                for (int j = 0; j < NB; ++j) rm[rr * G::LD + j] = v[j];
            }
            __syncwarp(mask);
#pragma unroll
            for (int j = 0; j < NB; ++j) {  // St_rj = (Q^H (R Q))_rj
                double2 s1 = mk(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NB; ++l) cfma(s1, cconj(q[l * G::LD + rr]), rm[l * G::LD + j]);
                v[j] = s1;
            }
        }
        __syncthreads();  // every read of Q is done: X takes its tile
        tile_load<NB>(sX, X + (size_t)k0 * G::NB2, nkt);
        __syncthreads();
        if (grp < nkt) {
            const int rr = r < NB ? r : 0;
            const bool live = r < NB;
            const double2* f = sF + grp * G::MS;
            double2* rm = sR + grp * G::MS;
            double2* x = sX + grp * G::MS;
#pragma unroll
            for (int j = 0; j < NB; ++j) {  // A_rj = ((Ft X)_rj - (X Ft)_rj) + St_rj
                double2 s2 = mk(0.0, 0.0), s3 = mk(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NB; ++l) {
                    cfma(s2, f[rr * G::LD + l], x[l * G::LD + j]);
                    cfma(s3, x[rr * G::LD + l], f[l * G::LD + j]);
                }
                v[j] = cadd(csub(s2, s3), v[j]);
            }
            __syncwarp(mask);
            const size_t kq = (size_t)(k0 + grp) * NB;
            const double wk = w[k0 + grp];
            const double dpr = sdp[grp * NB + rr], pr = sp[grp * NB + rr];
            if (live) {
#pragma unroll
                for (int j = 0; j < NB; ++j) rm[rr * G::LD + j] = v[j];
                const double pc = occ_clip(pr);
                double arr = v[0].x;
#pragma unroll
                for (int j = 1; j < NB; ++j)
                    if (j == rr) arr = v[j].x;
                const double hp = arr + T_r / (pc * (1.0 - pc)) * dpr;
                Hp[kq + rr] = hp;
                acc[1] += wk * dpr * hp;
                acc[2] += wk * dpr;
                acc[3] += wk * hp;
            }
            __syncwarp(mask);
            double2 hx[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                const double ddp = sdp[grp * NB + j] - dpr, dpp = sp[grp * NB + j] - pr;
                const double2 fij = f[rr * G::LD + j], fji = f[j * G::LD + rr];
                const double2 aij = rm[rr * G::LD + j], aji = rm[j * G::LD + rr];
                const double2 cij = mk(ddp * fij.x + dpp * aij.x, ddp * fij.y + dpp * aij.y);
                const double2 cji = mk(-ddp * fji.x - dpp * aji.x, -ddp * fji.y - dpp * aji.y);
                hx[j] = (j == rr) ? mk(0.0, 0.0) : mk(0.5 * (cij.x - cji.x), 0.5 * (cij.y + cji.y));
                if (live) {
                    const double2 xv = x[rr * G::LD + j];
                    acc[0] += xv.x * hx[j].x + xv.y * hx[j].y;
                }
            }
            __syncwarp(mask);
            if (live) {
#pragma unroll
                for (int j = 0; j < NB; ++j) x[rr * G::LD + j] = hx[j];
            }
        }
        __syncthreads();
        tile_store<NB>(HX + (size_t)k0 * G::NB2, sX, nkt);
        __syncthreads();
    }
    double out[4];
    if (reduce_last_block<4>(acc, R->part, &R->counter, out, red) && threadIdx.x == 0) {
        R->sums[kSumB1] = out[0];
        R->sums[kSumB2] = out[1];
        R->sums[kSumB3] = out[2];
        R->sums[kSumB4] = out[3];
    }
}

// ---------------------------------------------------------------------------
// Retraction Qt = Q U with U = (I - d/2)^{-1} (I + d/2), the Cayley factor at
// tau = -1 by elimination (equal to the spectral form V c(lam) V^H of
// solver_rtr.hpp:386-387), and ew = diag(U^H Ft U).
// Dynamic shared memory: sD | sQ | sF.
// ---------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(kThreads) k_rtr_retract_small(const double2* __restrict__ D,
                                                                const double2* __restrict__ Q,
                                                                const double2* __restrict__ Ft,
                                                                double2* __restrict__ Qt, double* __restrict__ ew,
                                                                int64_t nk) {
    using G = Geo<NB>;
    extern __shared__ __align__(16) double2 dyn[];
    double2* sD = dyn;
    double2* sQ = dyn + G::TILE;
    double2* sF = dyn + 2 * G::TILE;
    __shared__ double2 sPiv[G::KT * 4 * NB];
    const int grp = threadIdx.x / G::GS, r = threadIdx.x % G::GS;
    const unsigned mask = group_mask<NB>(threadIdx.x & 31);
    const int64_t ntiles = (nk + G::KT - 1) / G::KT;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t k0 = t * G::KT;
        const int nkt = (int)((nk - k0) < G::KT ? (nk - k0) : G::KT);
        tile_load<NB>(sD, D + (size_t)k0 * G::NB2, nkt);
        tile_load<NB>(sQ, Q + (size_t)k0 * G::NB2, nkt);
        tile_load<NB>(sF, Ft + (size_t)k0 * G::NB2, nkt);
        __syncthreads();
        if (grp < nkt) {
            const int rr = r < NB ? r : 0;
            const bool live = r < NB;
            double2* u = sD + grp * G::MS;
            double2* q = sQ + grp * G::MS;
            {
                double2 ur[NB];
                row_cayley<NB, G::LD>(u, -1.0, rr, sPiv + grp * 4 * NB, ur, mask);
                if (live) {
#pragma unroll
                    for (int j = 0; j < NB; ++j) u[rr * G::LD + j] = ur[j];
                }
            }
            __syncwarp(mask);
            {
                double2 qt[NB];
#pragma unroll
                for (int j = 0; j < NB; ++j) {  // (Q U)_rj
                    double2 a = mk(0.0, 0.0);
#pragma unroll
                    for (int l = 0; l < NB; ++l) cfma(a, q[rr * G::LD + l], u[l * G::LD + j]);
                    qt[j] = a;
                }
                __syncwarp(mask);
                if (live) {
#pragma unroll
                    for (int j = 0; j < NB; ++j) q[rr * G::LD + j] = qt[j];
                }
            }
            double2 ftj[NB];
#pragma unroll
            for (int l = 0; l < NB; ++l) ftj[l] = sF[grp * G::MS + rr * G::LD + l];
            const double er = row_diag_uhfu<NB, G::GS, G::LD>(ftj, u, r, mask, live);
            if (live) ew[(size_t)(k0 + grp) * NB + rr] = er;
        }
        __syncthreads();
        tile_store<NB>(Qt + (size_t)k0 * G::NB2, sQ, nkt);
        __syncthreads();
    }
}

template <int NB>
void rtr_small_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute(k_rtr_hvp_small<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(3 * sizeof(double2) * Geo<NB>::TILE));
        cudaFuncSetAttribute(k_rtr_retract_small<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(3 * sizeof(double2) * Geo<NB>::TILE));
        (void)cudaGetLastError();
    });
}

}  // namespace

bool rtr_small_supported(int nb) { return nb == 2 || nb == 4 || nb == 6 || nb == 8; }

int rtr_small_direction(const double2* rX, const double* rp, const double* eps, const double* p, const double* w,
                        const double2* Q, const double2* vX, const double* vp, double2* dX, double* dp, double2* dP,
                        int64_t nk, int nb, double T_r, double lam, double beta, double shift_z, double rz_old,
                        int mode, RtrScalars* R, cudaStream_t st) {
    const unsigned eg = flat_grid(nk * (int64_t)nb * nb, 256);  // one resident wave (4 x 256 threads per SM)
#define X(N)                                                                                                   \
    k_rtr_dir_elem<N><<<eg, 256, 0, st>>>(rX, rp, eps, p, w, vX, vp, dX, dp, nk, T_r, lam, beta, shift_z, rz_old, \
                                          mode, R);                                                            \
    CPPHF_LAUNCH_CHECK("rtr direction");                                                                       \
    k_rtr_dP_small<N><<<tiles_grid(nk, Geo<N>::KT, 16 * num_sms()), kThreads, 0, st>>>(Q, dX, dp, p, dP, nk);  \
    CPPHF_LAUNCH_CHECK("rtr density variation");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int rtr_small_hvp(const double2* Xd, const double* dp, const double2* Q, const double* p, const double2* Ft,
                  const double2* Fr, const double2* h, const double2* dP, const double* pen, const double* w,
                  double2* HX, double* Hp, int64_t nk, int nb, double T_r, RtrScalars* R, cudaStream_t st) {
#define X(N)                                                                                                     \
    rtr_small_attrs<N>();                                                                                        \
    k_rtr_hvp_small<N><<<tiles_grid(nk, Geo<N>::KT, kRtrMaxBlocks), kThreads,                                   \
                         3 * sizeof(double2) * Geo<N>::TILE, st>>>(Xd, dp, Q, p, Ft, Fr, h, dP, pen, w, HX, Hp, \
                                                                   nk, T_r, R);                                  \
    CPPHF_LAUNCH_CHECK("rtr hvp");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

int rtr_small_retract(const double2* D, const double2* Q, const double2* Ft, double2* Qt, double* ew, int64_t nk,
                      int nb, cudaStream_t st) {
#define X(N)                                                                                       \
    rtr_small_attrs<N>();                                                                          \
    k_rtr_retract_small<N><<<tiles_grid(nk, Geo<N>::KT, 16 * num_sms()), kThreads,                \
                             3 * sizeof(double2) * Geo<N>::TILE, st>>>(D, Q, Ft, Qt, ew, nk);      \
    CPPHF_LAUNCH_CHECK("rtr retract");
    SMALL_DISPATCH(nb, X)
#undef X
    return CPPHF_OK;
}

}  // namespace cpphf
