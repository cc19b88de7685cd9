// Trust-region Newton for HF direct minimisation on device-resident state
// (cpp_hf solver_rtr.hpp:163-459, optimizer "newton"), with the joint (Q, p)
// Hessian-vector product (solver_rtr.hpp:55-111) and the deflation bias
// (solver_rtr.hpp:124-157).
//
// The host replays the reference's control flow: every outer step runs a
// Steihaug truncated CG on the joint quadratic model (one Fock build of the
// linear response per Hessian-vector product), a Cayley retraction with
// tau = -1, the in-loop chemical-potential solve and one Fock build at the
// trial point, then the trust-region ratio test.  Every array operation is a
// kernel on the solve's stream; the host reads back only the scalars its
// decisions need (inner products, energies, gradient norms).
//
// Vectors never materialised: the preconditioned residual z is formed from r
// where it is used (its occupation part's weighted mean is removed through the
// host-side scalar shift), and the projection of the Hessian's occupation part
// onto the particle-conserving subspace is applied as a scalar shift inside
// the kernels that read it.  The current and trial states live in two slots
// (Q, p, Ft, G, eps, mu, energy, deflation curvature) so that accepting or
// rejecting a step swaps an index instead of copying fields.
#include "common.cuh"
#include "dm.cuh"
#include "dm_small.cuh"
#include "eigh.cuh"
#include "fock.cuh"
#include "mu.cuh"
#include "rtr.cuh"
#include "solve_util.cuh"
#include "team.cuh"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

namespace cpphf {

namespace {

constexpr int kRtrMaxNb = 48;    // five team matrices per k-point in shared memory
constexpr int kMaxDeflation = 256;
constexpr double kTinyReal = 1.0e-30;

unsigned flat_blocks(int64_t n, int threads) {
    const int64_t want = (n + threads - 1) / threads;
    const int64_t cap = std::min<int64_t>((int64_t)num_sms() * 4, kRtrMaxBlocks);
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, cap));
}

TeamLaunch rtr_team_launch(int64_t nk, int nb) {
    TeamLaunch L = team_launch(nk, nb);
    L.grid = std::min<unsigned>(L.grid, kRtrMaxBlocks);
    return L;
}

__global__ void k_rtr_wsum(const double* __restrict__ w, int64_t nk, RtrScalars* R) {
    __shared__ double red[32];
    double v[1] = {0.0};
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += (int64_t)gridDim.x * blockDim.x)
        v[0] += w[k];
    double out[1];
    if (reduce_last_block<1>(v, R->part, &R->counter, out, red) && threadIdx.x == 0) R->sums[kSumW] = out[0];
}

// ---------------------------------------------------------------------------
// Direction and its density variation (solver_rtr.hpp:61-75, 218-231, 356-362).
// mode 0: d = z(r); mode 1: d = z(r) + beta d; mode 2: d given; mode 3: as 1
// with beta and shift_z formed here from the update pass's sums.  z(r) is the
// block preconditioner: rX / sqrt(gap^2 + lam^2) and rp p(1-p) / T minus the
// weighted mean shift_z.  Then dP = herm(Q M Q^H) with M = [X, diag p]
// off the diagonal and dp on it.  Sums <d,d>, <v,d>, <v,v> in the joint metric
// (orbital part unweighted, occupation part w2d-weighted).
// ---------------------------------------------------------------------------
template <bool WARP>
__global__ void k_rtr_direction(const double2* __restrict__ rX, const double* __restrict__ rp,
                                const double* __restrict__ eps, const double* __restrict__ p,
                                const double* __restrict__ w, const double2* __restrict__ Q,
                                const double2* __restrict__ vX, const double* __restrict__ vp, double2* dX,
                                double* dp, double2* __restrict__ dP, int64_t nk, int nb, double T_r, double lam,
                                double beta, double shift_z, double rz_old, int mode, RtrScalars* R) {
    extern __shared__ __align__(16) unsigned char raw[];
    __shared__ double red[32 * 3];
    Team<WARP> t;
    const int ld = nb + 1, nb2 = nb * nb;
    double2* sQ = team_mats<WARP>(raw, nb, 3, nb, t.team);
    double2* sM = sQ + team_mat_elems(nb);
    double2* sT = sM + team_mat_elems(nb);
    double* sdp = reinterpret_cast<double*>(sT + team_mat_elems(nb));
    const double lam2 = lam * lam;
    if (mode == 3) {  // beta and shift_z from the preceding update pass (same arithmetic as the host)
        const double den = R->sums[kSumW] * (double)nb;
        shift_z = den > 0.0 ? R->sums[kSumA3] / den : 0.0;
        beta = (R->sums[kSumA1] + R->sums[kSumA2] - shift_z * R->sums[kSumA4]) / rz_old;
        mode = 1;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(sQ, Q + (size_t)k * nb2, nb, t);
        const double* pk = p + (size_t)k * nb;
        const double wk = w[k];
        for (int b = t.tid; b < nb; b += t.nt) {
            const size_t q = (size_t)k * nb + b;
            double d;
            if (mode == 2) {
                d = dp[q];
            } else {
                const double pc = occ_clip(pk[b]);
                const double z = rp[q] * pc * (1.0 - pc) / T_r - shift_z;
                d = mode == 0 ? z : z + beta * dp[q];
                dp[q] = d;
            }
            sdp[b] = d;
            acc[0] += wk * d * d;
            if (vp) {
                const double v = vp[q];
                acc[1] += wk * v * d;
                acc[2] += wk * v * v;
            }
        }
        t.sync();
        const double* ek = eps ? eps + (size_t)k * nb : nullptr;
        for (int e = t.tid; e < nb2; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            const size_t g = (size_t)k * nb2 + e;
            double2 d;
            if (mode == 2) {
                d = dX[g];
            } else {
                const double gap = ek[i] - ek[j];
                const double s = sqrt(gap * gap + lam2);
                const double2 r = rX[g];
                d = mk(r.x / s, r.y / s);
                if (mode == 1) {
                    const double2 o = dX[g];
                    d = mk(d.x + beta * o.x, d.y + beta * o.y);
                }
                dX[g] = d;
            }
            acc[0] += d.x * d.x + d.y * d.y;
            if (vX) {
                const double2 v = vX[g];
                acc[1] += v.x * d.x + v.y * d.y;
                acc[2] += v.x * v.x + v.y * v.y;
            }
            sM[i * ld + j] = (i == j) ? mk(sdp[i], 0.0) : cscale(d, pk[j] - pk[i]);
        }
        t.sync();
        tmm<false, false, WARP>(sT, sQ, sM, nb, t);  // Q M
        t.sync();
        tmm<false, true, WARP>(sM, sT, sQ, nb, t);   // (Q M) Q^H
        t.sync();
        for (int e = t.tid; e < nb2; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            const double2 a = sM[i * ld + j], b = sM[j * ld + i];
            dP[(size_t)k * nb2 + e] = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        }
        t.sync();
    }
    double out[3];
    if (reduce_last_block<3>(acc, R->part, &R->counter, out, red) && threadIdx.x == 0) {
        R->sums[kSumDD] = out[0];
        R->sums[kSumVD] = out[1];
        R->sums[kSumVV] = out[2];
    }
}

// ---------------------------------------------------------------------------
// Hessian-vector product assembly (solver_rtr.hpp:86-109): R = F[dP] - h
// (+ pen dP), St = Q^H R Q, A = Ft X - X Ft + St,
// C_ij = (dp_j - dp_i) Ft_ij + (p_j - p_i) A_ij, HX = (C - C^H)/2 with a zero
// diagonal, Hp_b = Re A_bb + T / (pc (1 - pc)) dp_b (before the projection,
// which the caller applies from the sums B4 / (nb sum w)).
// ---------------------------------------------------------------------------
template <bool WARP>
__global__ void k_rtr_hvp(const double2* __restrict__ X, const double* __restrict__ dp,
                          const double2* __restrict__ Q, const double* __restrict__ p,
                          const double2* __restrict__ Ft, const double2* __restrict__ Fr,
                          const double2* __restrict__ h, const double2* __restrict__ dP,
                          const double* __restrict__ pen, const double* __restrict__ w, double2* __restrict__ HX,
                          double* __restrict__ Hp, int64_t nk, int nb, double T_r, RtrScalars* R) {
    extern __shared__ __align__(16) unsigned char raw[];
    __shared__ double red[32 * 4];
    Team<WARP> t;
    const int ld = nb + 1, nb2 = nb * nb;
    const size_t me = team_mat_elems(nb);
    double2* sQ = team_mats<WARP>(raw, nb, 5, 2 * nb, t.team);
    double2* sF = sQ + me;
    double2* sX = sF + me;
    double2* sR = sX + me;
    double2* sT = sR + me;
    double* sdp = reinterpret_cast<double*>(sT + me);
    double* sp = sdp + nb;
    const double pc_ = pen ? *pen : 0.0;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        const size_t o = (size_t)k * nb2;
        tload<WARP>(sQ, Q + o, nb, t);
        tload<WARP>(sF, Ft + o, nb, t);
        tload<WARP>(sX, X + o, nb, t);
        for (int e = t.tid; e < nb2; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            double2 r = csub(Fr[o + e], h[o + e]);
            if (pc_ != 0.0) {
                const double2 d = dP[o + e];
                r = mk(r.x + pc_ * d.x, r.y + pc_ * d.y);
            }
            sR[i * ld + j] = r;
        }
        for (int b = t.tid; b < nb; b += t.nt) {
            sdp[b] = dp[(size_t)k * nb + b];
            sp[b] = p[(size_t)k * nb + b];
        }
        t.sync();
        tmm<false, false, WARP>(sT, sR, sQ, nb, t);  // R Q
        t.sync();
        tmm<true, false, WARP>(sR, sQ, sT, nb, t);   // St = Q^H (R Q)
        t.sync();
        for (int e = t.tid; e < nb2; e += t.nt) {  // A = Ft X - X Ft + St
            const int i = e / nb, j = e - i * nb;
            double2 a1 = mk(0.0, 0.0), a2 = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) {
                cfma(a1, sF[i * ld + l], sX[l * ld + j]);
                cfma(a2, sX[i * ld + l], sF[l * ld + j]);
            }
            sT[i * ld + j] = cadd(csub(a1, a2), sR[i * ld + j]);
        }
        t.sync();
        const double wk = w[k];
        for (int e = t.tid; e < nb2; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            double2 hx = mk(0.0, 0.0);
            if (i != j) {
                const double2 fij = sF[i * ld + j], fji = sF[j * ld + i];
                const double2 aij = sT[i * ld + j], aji = sT[j * ld + i];
                const double ddp = sdp[j] - sdp[i], dpp = sp[j] - sp[i];
                const double2 cij = mk(ddp * fij.x + dpp * aij.x, ddp * fij.y + dpp * aij.y);
                const double2 cji = mk(-ddp * fji.x - dpp * aji.x, -ddp * fji.y - dpp * aji.y);
                hx = mk(0.5 * (cij.x - cji.x), 0.5 * (cij.y + cji.y));
            }
            HX[o + e] = hx;
            const double2 x = sX[i * ld + j];
            acc[0] += x.x * hx.x + x.y * hx.y;
        }
        for (int b = t.tid; b < nb; b += t.nt) {
            const double pc = occ_clip(sp[b]);
            const double hp = sT[b * ld + b].x + T_r / (pc * (1.0 - pc)) * sdp[b];
            Hp[(size_t)k * nb + b] = hp;
            acc[1] += wk * sdp[b] * hp;
            acc[2] += wk * sdp[b];
            acc[3] += wk * hp;
        }
        t.sync();
    }
    double out[4];
    if (reduce_last_block<4>(acc, R->part, &R->counter, out, red) && threadIdx.x == 0) {
        R->sums[kSumB1] = out[0];
        R->sums[kSumB2] = out[1];
        R->sums[kSumB3] = out[2];
        R->sums[kSumB4] = out[3];
    }
}

// Hp -= sum_k w_k sum_b Hp / (nb sum_k w_k)   (project_occ, solver_rtr.hpp:42-50)
__global__ void k_rtr_project_occ(double* Hp, int64_t n, int nb, const RtrScalars* R) {
    const double den = R->sums[kSumW] * (double)nb;
    const double shift = den > 0.0 ? R->sums[kSumB4] / den : 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        Hp[i] -= shift;
}

// ---------------------------------------------------------------------------
// CG vector updates (solver_rtr.hpp:304-364).  mode 0: v += a d, Hv += a Hd,
// r -= a Hd; mode 1 (to the trust-region boundary): v += a d, Hv += a Hd;
// mode 2 (start): r = -G, v = Hv = 0.  Hd's occupation part is shifted by
// shift_h (its projection).  Modes 0 and 2 then reduce over the new r:
// <r,r>, Re<rX, zX>, sum w rp z, sum w z, sum w rp with z = rp p(1-p)/T.
// ---------------------------------------------------------------------------
__global__ void k_rtr_update(int mode, double a, double shift_h, const double2* __restrict__ G, double2* vX,
                             double2* HvX, double2* rX, const double2* __restrict__ dX,
                             const double2* __restrict__ HDX, double* vp, double* Hvp, double* rp,
                             const double* __restrict__ dp, const double* __restrict__ HDp,
                             const double* __restrict__ eps, const double* __restrict__ p,
                             const double* __restrict__ w, int64_t nk, int nb, double T_r, double lam,
                             RtrScalars* R) {
    __shared__ double red[32 * 5];
    const int nb2 = nb * nb;
    const int64_t n_orb = nk * nb2, n_occ = nk * nb;
    const double lam2 = lam * lam;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_orb; e += stride) {
        double2 r;
        if (mode == 2) {
            r = mk(-G[e].x, -G[e].y);
            rX[e] = r;
            vX[e] = mk(0.0, 0.0);
            HvX[e] = mk(0.0, 0.0);
        } else {
            const double2 d = dX[e], hd = HDX[e];
            const double2 v = vX[e], hv = HvX[e];
            vX[e] = mk(v.x + a * d.x, v.y + a * d.y);
            HvX[e] = mk(hv.x + a * hd.x, hv.y + a * hd.y);
            if (mode == 1) continue;
            const double2 ro = rX[e];
            r = mk(ro.x - a * hd.x, ro.y - a * hd.y);
            rX[e] = r;
        }
        const int64_t k = e / nb2;
        const int rem = (int)(e - k * nb2), i = rem / nb, j = rem - i * nb;
        const double gap = eps[k * nb + i] - eps[k * nb + j];
        const double s = sqrt(gap * gap + lam2);
        const double rr = r.x * r.x + r.y * r.y;
        acc[0] += rr;
        acc[1] += r.x * (r.x / s) + r.y * (r.y / s);
    }
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n_occ; q += stride) {
        double r;
        if (mode == 2) {
            r = 0.0;
            rp[q] = 0.0;
            vp[q] = 0.0;
            Hvp[q] = 0.0;
        } else {
            const double d = dp[q], hd = HDp[q] - shift_h;
            vp[q] += a * d;
            Hvp[q] += a * hd;
            if (mode == 1) continue;
            r = rp[q] - a * hd;
            rp[q] = r;
        }
        const double wk = w[q / nb];
        const double pc = occ_clip(p[q]);
        const double z = r * pc * (1.0 - pc) / T_r;
        acc[0] += wk * r * r;
        acc[2] += wk * r * z;
        acc[3] += wk * z;
        acc[4] += wk * r;
    }
    if (mode == 1) return;
    double out[5];
    if (reduce_last_block<5>(acc, R->part, &R->counter, out, red) && threadIdx.x == 0) {
        R->sums[kSumRR] = out[0];
        R->sums[kSumA1] = out[1];
        R->sums[kSumA2] = out[2];
        R->sums[kSumA3] = out[3];
        R->sums[kSumA4] = out[4];
    }
}

// Predicted-reduction terms (solver_rtr.hpp:376-378) and |v| in the joint metric:
// sum w Re<G, vX>, sum w Re<vX, HvX>, sum w vp Hvp, sum |vX|^2, sum w vp^2.
__global__ void k_rtr_model(const double2* __restrict__ G, const double2* __restrict__ vX,
                            const double2* __restrict__ HvX, const double* __restrict__ vp,
                            const double* __restrict__ Hvp, const double* __restrict__ w, int64_t nk, int nb,
                            RtrScalars* R) {
    __shared__ double red[32 * 5];
    const int nb2 = nb * nb;
    const int64_t n_orb = nk * nb2, n_occ = nk * nb;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_orb; e += stride) {
        const double wk = w[e / nb2];
        const double2 g = G[e], v = vX[e], hv = HvX[e];
        acc[0] += wk * (g.x * v.x + g.y * v.y);
        acc[1] += wk * (v.x * hv.x + v.y * hv.y);
        acc[3] += v.x * v.x + v.y * v.y;
    }
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n_occ; q += stride) {
        const double wk = w[q / nb];
        acc[2] += wk * vp[q] * Hvp[q];
        acc[4] += wk * vp[q] * vp[q];
    }
    double out[5];
    if (reduce_last_block<5>(acc, R->part, &R->counter, out, red) && threadIdx.x == 0) {
        R->sums[kSumGV] = out[0];
        R->sums[kSumVHX] = out[1];
        R->sums[kSumVHP] = out[2];
        R->sums[kSumVVX] = out[3];
        R->sums[kSumVVP] = out[4];
    }
}

// ---------------------------------------------------------------------------
// Retraction (solver_rtr.hpp:380-396): U = V diag(c) V^H with the Cayley factor
// c = (1 + i tau lam / 2) / (1 - i tau lam / 2) at tau = -1, Qt = Q U, and the
// trial orbital energies diag(U^H Ft U) from the frozen Ft.
// ---------------------------------------------------------------------------
template <bool WARP>
__global__ void k_rtr_retract(const double2* __restrict__ V, const double* __restrict__ lam,
                              const double2* __restrict__ Q, const double2* __restrict__ Ft,
                              double2* __restrict__ Qt, double* __restrict__ ew, int64_t nk, int nb) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    const int ld = nb + 1, nb2 = nb * nb;
    const size_t me = team_mat_elems(nb);
    double2* sV = team_mats<WARP>(raw, nb, 4, 2 * nb, t.team);
    double2* sU = sV + me;
    double2* sQ = sU + me;
    double2* sF = sQ + me;
    double2* sc = sF + me;
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        const size_t o = (size_t)k * nb2;
        tload<WARP>(sV, V + o, nb, t);
        tload<WARP>(sQ, Q + o, nb, t);
        tload<WARP>(sF, Ft + o, nb, t);
        for (int b = t.tid; b < nb; b += t.nt) sc[b] = cayley_factor(lam[(size_t)k * nb + b], -1.0);
        t.sync();
        for (int e = t.tid; e < nb2; e += t.nt) {  // U_ij = sum_b V_ib c_b conj(V_jb)
            const int i = e / nb, j = e - i * nb;
            double2 acc = mk(0.0, 0.0);
            for (int b = 0; b < nb; ++b) cfma(acc, cmul(sV[i * ld + b], sc[b]), cconj(sV[j * ld + b]));
            sU[i * ld + j] = acc;
        }
        t.sync();
        for (int e = t.tid; e < nb2; e += t.nt) {  // Qt = Q U;  W = Ft U (into sV)
            const int i = e / nb, j = e - i * nb;
            double2 q = mk(0.0, 0.0), f = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) {
                cfma(q, sQ[i * ld + l], sU[l * ld + j]);
                cfma(f, sF[i * ld + l], sU[l * ld + j]);
            }
            Qt[o + e] = q;
            sV[i * ld + j] = f;
        }
        t.sync();
        for (int b = t.tid; b < nb; b += t.nt) {  // Re (U^H W)_bb
            double s = 0.0;
            for (int l = 0; l < nb; ++l) {
                const double2 u = sU[l * ld + b], f = sV[l * ld + b];
                s += u.x * f.x + u.y * f.y;
            }
            ew[(size_t)k * nb + b] = s;
        }
        t.sync();
    }
}

// ---------------------------------------------------------------------------
// Deflation bias (solver_rtr.hpp:124-157)
// ---------------------------------------------------------------------------
__global__ void k_defl_dist(const double2* __restrict__ P, const double2* __restrict__ T,
                            const double* __restrict__ w, int64_t nk, int nb2, double* d2, RtrScalars* R) {
    __shared__ double red[32];
    const int64_t n = nk * nb2;
    double acc[1] = {0.0};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 d = csub(P[e], T[e]);
        acc[0] += w[e / nb2] * (d.x * d.x + d.y * d.y);
    }
    double out[1];
    if (reduce_last_block<1>(acc, R->part, &R->counter, out, red) && threadIdx.x == 0) *d2 = out[0];
}

// out = base + sum_i 2 phi'(d_i^2) (P - T_i), phi(x) = sigma exp(-x / (2 L^2));
// block 0 writes Phi and 2 sum_i phi'(d_i^2), and adds Phi to *energy.
__global__ void k_defl_apply(const double2* __restrict__ P, const double2* __restrict__ targets, int n_defl,
                             int64_t n, const double* __restrict__ d2, double sigma, double inv2L2,
                             const double2* base, double2* out, double* energy, double* phi_out,
                             double* pen_out) {
    __shared__ double coeff[kMaxDeflation];
    for (int i = threadIdx.x; i < n_defl; i += blockDim.x) {
        const double phi = sigma * exp(-d2[i] * inv2L2);
        coeff[i] = 2.0 * (-phi * inv2L2);
    }
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double Phi = 0.0, diag = 0.0;
        for (int i = 0; i < n_defl; ++i) {
            const double phi = sigma * exp(-d2[i] * inv2L2);
            Phi += phi;
            diag += -phi * inv2L2;
        }
        if (phi_out) *phi_out = Phi;
        if (pen_out) *pen_out = 2.0 * diag;
        if (energy) *energy += Phi;
    }
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 pe = P[e];
        double2 s = mk(0.0, 0.0);
        for (int i = 0; i < n_defl; ++i) {
            const double2 d = csub(pe, targets[(size_t)i * n + e]);
            s = mk(s.x + coeff[i] * d.x, s.y + coeff[i] * d.y);
        }
        out[e] = base ? cadd(base[e], s) : s;
    }
}

template <class F>
void set_smem_once(F f) {
    raise_smem(f);
}

void init_rtr_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        set_smem_once(k_rtr_direction<true>);
        set_smem_once(k_rtr_direction<false>);
        set_smem_once(k_rtr_hvp<true>);
        set_smem_once(k_rtr_hvp<false>);
        set_smem_once(k_rtr_retract<true>);
        set_smem_once(k_rtr_retract<false>);
    });
}

int rtr_check_nb(int64_t nb) {
    if (nb < 1) return fail(CPPHF_ERR_INVALID, "nb must be positive");
    if (nb > kRtrMaxNb) return fail(CPPHF_ERR_UNSUPPORTED, "trust-region Newton supports nb <= 48");
    return CPPHF_OK;
}

int launch_direction(const double2* rX, const double* rp, const double* eps, const double* p, const double* w,
                     const double2* Q, const double2* vX, const double* vp, double2* dX, double* dp, double2* dP,
                     int64_t nk, int nb, double T_r, double lam, double beta, double shift_z, double rz_old,
                     int mode, RtrScalars* R, cudaStream_t st) {
    if (rtr_small_supported(nb))
        return rtr_small_direction(rX, rp, eps, p, w, Q, vX, vp, dX, dp, dP, nk, nb, T_r, lam, beta, shift_z, rz_old,
                                   mode, R, st);
    const TeamLaunch L = rtr_team_launch(nk, nb);
    TEAM_DISPATCH(L, k_rtr_direction, 3, nb, rX, rp, eps, p, w, Q, vX, vp, dX, dp, dP, nk, nb, T_r, lam, beta,
                  shift_z, rz_old, mode, R);
    return CPPHF_OK;
}

int launch_hvp(const double2* X, const double* dp, const double2* Q, const double* p, const double2* Ft,
               const double2* Fr, const double2* h, const double2* dP, const double* pen, const double* w,
               double2* HX, double* Hp, int64_t nk, int nb, double T_r, RtrScalars* R, cudaStream_t st) {
    if (rtr_small_supported(nb)) return rtr_small_hvp(X, dp, Q, p, Ft, Fr, h, dP, pen, w, HX, Hp, nk, nb, T_r, R, st);
    const TeamLaunch L = rtr_team_launch(nk, nb);
    TEAM_DISPATCH(L, k_rtr_hvp, 5, 2 * nb, X, dp, Q, p, Ft, Fr, h, dP, pen, w, HX, Hp, nk, nb, T_r, R);
    return CPPHF_OK;
}

int launch_retract(const double2* V, const double* lam, const double2* Q, const double2* Ft, double2* Qt,
                   double* ew, int64_t nk, int nb, cudaStream_t st) {
    const TeamLaunch L = team_launch(nk, nb);
    TEAM_DISPATCH(L, k_rtr_retract, 4, 2 * nb, V, lam, Q, Ft, Qt, ew, nk, nb);
    return CPPHF_OK;
}

// Phi, S_pen (added to `base` when given) and the curvature of the deflation
// bias at P; d2 holds n_defl doubles of scratch.
int deflation(const double2* P, const double2* targets, int64_t n_defl, const double* w, int64_t nk, int nb,
              double sigma, double length, const double2* base, double2* out, double* energy, double* phi_out,
              double* pen_out, double* d2, RtrScalars* R, cudaStream_t st) {
    const int64_t n = nk * (int64_t)nb * nb;
    const unsigned fg = flat_blocks(n, 256);
    for (int64_t i = 0; i < n_defl; ++i) {
        k_defl_dist<<<fg, 256, 0, st>>>(P, targets + (size_t)i * n, w, nk, nb * nb, d2 + i, R);
        CPPHF_LAUNCH_CHECK("deflation distance");
    }
    const double inv2L2 = 1.0 / (2.0 * length * length);
    k_defl_apply<<<fg, 256, 0, st>>>(P, targets, (int)n_defl, n, d2, sigma, inv2L2, base, out, energy, phi_out,
                                     pen_out);
    CPPHF_LAUNCH_CHECK("deflation bias");
    return CPPHF_OK;
}

struct RtrLayout {
    size_t Q[2], Ft[2], G[2], P, Sig, F, vX, HvX, rX, dX, HDX, dP, Vd;
    size_t p[2], eps[2], gp, ew, lamd, vp, Hvp, rp, dp, HDp, wn;
    size_t S, R, d2, fock_ws, mu_ws, pack, total;
    size_t fock_bytes, mu_bytes;
};

size_t fock_bytes_rtr(const cpphf_kernel* K) {
    // the response build runs without the reference density, the state builds with it
    cpphf_kernel Kr = *K;
    Kr.has_refP = 0;
    return std::max(fock_bytes_packed_kernel(K), fock_bytes_packed_kernel(&Kr));
}

RtrLayout rtr_layout(const cpphf_kernel* K, int64_t n_defl) {
    const size_t nk = (size_t)K->nk1 * K->nk2, nb = (size_t)K->nb;
    const size_t fld = sizeof(double2) * nk * nb * nb, vec = sizeof(double) * nk * nb;
    struct Take {
        size_t total = 0;
        size_t operator()(size_t bytes) {
            const size_t at = total;
            total += (bytes + 255) & ~(size_t)255;
            return at;
        }
    } take;
    RtrLayout L;
    for (int s = 0; s < 2; ++s) {
        L.Q[s] = take(fld);
        L.Ft[s] = take(fld);
        L.G[s] = take(fld);
        L.p[s] = take(vec);
        L.eps[s] = take(vec);
    }
    L.P = take(fld);
    L.Sig = take(fld);
    L.F = take(fld);
    L.vX = take(fld);
    L.HvX = take(fld);
    L.rX = take(fld);
    L.dX = take(fld);
    L.HDX = take(fld);
    L.dP = take(fld);
    L.Vd = take(fld);
    L.gp = take(vec);
    L.ew = take(vec);
    L.lamd = take(vec);
    L.vp = take(vec);
    L.Hvp = take(vec);
    L.rp = take(vec);
    L.dp = take(vec);
    L.HDp = take(vec);
    L.wn = take(sizeof(double) * nk);
    L.S = take(sizeof(DmScalars));
    L.R = take(sizeof(RtrScalars));
    L.d2 = take(sizeof(double) * (size_t)std::max<int64_t>(n_defl, 1));
    L.fock_bytes = fock_bytes_rtr(K);
    L.fock_ws = take(L.fock_bytes);
    L.mu_bytes = mu_workspace_bytes((int64_t)nk, (int64_t)nb);
    L.mu_ws = take(L.mu_bytes);
    L.pack = take(solver_pack_bytes(K));
    L.total = take.total;
    return L;
}

bool deflation_on(const cpphf_dm_config* cfg) {
    return cfg->n_deflation > 0 && cfg->deflation_sigma > 0.0 && cfg->deflation_targets != nullptr;
}

}  // namespace

size_t solve_rtr_workspace_bytes(const cpphf_kernel* K, const cpphf_dm_config* cfg) {
    return rtr_layout(K, deflation_on(cfg) ? cfg->n_deflation : 0).total;
}

int solve_rtr(const cpphf_kernel* K, const cpphf_dm_config* cfg, const double2* P0, double n_e,
              cpphf_project_fn project, void* puser, double2* Q_out, double* p_out, double2* D_out, double2* F_out,
              double* hist_E, double* hist_G, cpphf_dm_result* res, void* ws, size_t wsb, cudaStream_t st) {
    CPPHF_TRY(rtr_check_nb(K->nb));
    const bool defl = deflation_on(cfg);
    if (defl && cfg->n_deflation > kMaxDeflation)
        return fail(CPPHF_ERR_UNSUPPORTED, "more than 256 deflation targets");
    if (cfg->tr_cg_max < 0) return fail(CPPHF_ERR_INVALID, "tr_cg_max must be >= 0");
    const RtrLayout L = rtr_layout(K, defl ? cfg->n_deflation : 0);
    if (!ws || wsb < L.total)
        return fail(CPPHF_ERR_INVALID,
                    "solve_dm (newton): workspace too small (" + std::to_string(L.total) + " bytes needed)");
    init_rtr_attrs();
    unsigned char* W = static_cast<unsigned char*>(ws);
    cpphf_kernel Kp;  // K with its packed VR / h (Hermitian packing), made once per solve
    CPPHF_TRY(solver_pack(K, &Kp, W + L.pack, st));
    K = &Kp;
    auto fld = [&](size_t off) { return reinterpret_cast<double2*>(W + off); };
    auto vec = [&](size_t off) { return reinterpret_cast<double*>(W + off); };
    double2* Q[2] = {fld(L.Q[0]), fld(L.Q[1])};
    double2* Ft[2] = {fld(L.Ft[0]), fld(L.Ft[1])};
    double2* G[2] = {fld(L.G[0]), fld(L.G[1])};
    double* p[2] = {vec(L.p[0]), vec(L.p[1])};
    double* eps[2] = {vec(L.eps[0]), vec(L.eps[1])};
    double2 *P = fld(L.P), *Sig = fld(L.Sig), *F = fld(L.F), *vX = fld(L.vX), *HvX = fld(L.HvX), *rX = fld(L.rX),
            *dX = fld(L.dX), *HDX = fld(L.HDX), *dP = fld(L.dP), *Vd = fld(L.Vd);
    double *gp = vec(L.gp), *ew = vec(L.ew), *lamd = vec(L.lamd), *vp = vec(L.vp), *Hvp = vec(L.Hvp),
           *rp = vec(L.rp), *dp = vec(L.dp), *HDp = vec(L.HDp), *wn = vec(L.wn), *d2 = vec(L.d2);
    DmScalars* S = reinterpret_cast<DmScalars*>(W + L.S);
    RtrScalars* R = reinterpret_cast<RtrScalars*>(W + L.R);
    void* fws = W + L.fock_ws;
    void* mws = W + L.mu_ws;
    const double2* targets = static_cast<const double2*>(cfg->deflation_targets);

    const int64_t nk = K->nk1 * K->nk2;
    const int nb = (int)K->nb;
    const int64_t npb = nk * nb;
    const size_t fbytes = sizeof(double2) * (size_t)nk * nb * nb, vbytes = sizeof(double) * (size_t)npb;
    const double wsum = std::max(K->weight_sum, kTinyReal);
    const double n_t = n_e / wsum;
    const double T_r = std::max(K->T, 1.0e-12);
    const double tol_g = cfg->tol_grad > 0.0 ? cfg->tol_grad : 1.0e-6;
    const int64_t max_iter = std::max<int64_t>(0, cfg->max_iter);
    const int mu_it = cfg->mu_maxiter;
    const double d_len = std::max(cfg->deflation_length, 1.0e-12);
    const bool small = dm_small_supported(nb);
    cpphf_kernel Kr = *K;  // linear response: no reference-density subtraction (solver_rtr.hpp:35)
    Kr.has_refP = 0;

    CPPHF_CUDA(cudaMemsetAsync(S, 0, sizeof(DmScalars), st));
    CPPHF_CUDA(cudaMemsetAsync(R, 0, sizeof(RtrScalars), st));
    CPPHF_TRY(scale_weights(K->w2d, wsum, wn, nk, st));
    k_rtr_wsum<<<flat_blocks(nk, 256), 256, 0, st>>>(K->w2d, nk, R);
    CPPHF_LAUNCH_CHECK("rtr weight sum");

    // occupations p[s] = expit((mu[s] - e) / T) and the density P = Q diag(p) Q^H
    auto occupy = [&](int s, const double* e) -> int {
        if (small) return dm_small_dens_occ(Q[s], e, &R->mu[s], T_r, p[s], P, nk, nb, st);
        CPPHF_TRY(dm_occupations(e, &R->mu[s], T_r, p[s], npb, st));
        return dm_density(Q[s], p[s], P, nk, nb, st);
    };
    auto finish_density = [&]() -> int {
        if (project) {
            CPPHF_TRY(call_project(project, puser, P, K, st));
            CPPHF_TRY(hermitize(P, P, nk, nb, st));
        }
        return CPPHF_OK;
    };
    // eval_state (solver_rtr.hpp:264-285) of slot s from the density in P:
    // energy (+ bias), Ft = Q^H (F + S_pen) Q, eps = diag Ft, gradient G and its
    // norm, and the preconditioner scale lam_pc (solver_rtr.hpp:300-302)
    double hE[2] = {0.0, 0.0}, hg[2] = {0.0, 0.0}, hlam[2] = {0.0, 0.0};
    double* const hb = host_scalars();  // pinned scalar read-back: hb[0..3], then the sums
    double* const sums = hb + 8;
    static_assert(8 + kNumSums <= kHostScalars, "host scalar layout");
    auto eval = [&](int s, bool with_model) -> int {
        CPPHF_TRY(finish_density());
        CPPHF_TRY(build_fock(K, P, solver_sigma(K, Sig), Ft[s], nullptr, &R->energy[s], nullptr, fws, L.fock_bytes, st));
        if (defl)
            CPPHF_TRY(deflation(P, targets, cfg->n_deflation, K->w2d, nk, nb, cfg->deflation_sigma, d_len, Ft[s],
                                Ft[s], &R->energy[s], &R->phi, &R->pen[s], d2, R, st));
        if (small) {
            CPPHF_TRY(dm_small_rot_grad(Q[s], Ft[s], p[s], wn, eps[s], G[s], gp, nk, nb, T_r, cfg->denom_scale, S,
                                        st));
        } else {
            CPPHF_TRY(dm_rotate(Q[s], Ft[s], Ft[s], eps[s], nk, nb, st));
            CPPHF_TRY(dm_gradient(Ft[s], p[s], eps[s], wn, G[s], gp, nk, nb, T_r, cfg->denom_scale, S, st));
        }
        CPPHF_CUDA(cudaMemcpyAsync(hb, &R->mu[s], sizeof(double), cudaMemcpyDeviceToHost, st));
        CPPHF_CUDA(cudaMemcpyAsync(hb + 1, &R->energy[s], sizeof(double), cudaMemcpyDeviceToHost, st));
        static_assert(offsetof(DmScalars, lam_pc) == offsetof(DmScalars, grad_norm) + sizeof(double),
                      "DmScalars read-back layout");
        CPPHF_CUDA(cudaMemcpyAsync(hb + 2, &S->grad_norm, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (with_model)
            CPPHF_CUDA(cudaMemcpyAsync(sums + kSumGV, &R->sums[kSumGV], 5 * sizeof(double), cudaMemcpyDeviceToHost,
                                       st));
        CPPHF_CUDA(cudaStreamSynchronize(st));
        if (!std::isfinite(hb[0]))
            return fail(CPPHF_ERR_TIMEOUT,
                        "solve_dm (newton): chemical-potential solve failed (device wait timeout or non-finite)");
        hE[s] = hb[1];
        hg[s] = hb[2];
        hlam[s] = hb[3];
        return CPPHF_OK;
    };
    auto read_sums = [&](int first, int count) -> int {
        CPPHF_CUDA(cudaMemcpyAsync(sums + first, &R->sums[first], sizeof(double) * count, cudaMemcpyDeviceToHost,
                                   st));
        CPPHF_CUDA(cudaStreamSynchronize(st));
        return CPPHF_OK;
    };

    // ---- initialise (Q, p) from F[P0] (solver_rtr.hpp:251-262) ----
    CPPHF_TRY(hermitize(P0, P, nk, nb, st));
    CPPHF_TRY(build_fock(K, P, solver_sigma(K, Sig), F, nullptr, nullptr, nullptr, fws, L.fock_bytes, st));
    CPPHF_TRY(eigh_batched(F, eps[0], Q[0], nk, nb, 0, nullptr, st));
    CPPHF_TRY(mu_solve(eps[0], wn, nk, nb, n_t, &R->mu[0], T_r, mu_it, 1, &R->mu[0], mws, L.mu_bytes, st));
    CPPHF_TRY(occupy(0, eps[0]));
    CPPHF_TRY(eval(0, false));
    CPPHF_TRY(read_sums(kSumW, 1));
    const double wtot = sums[kSumW];
    const double occ_den = wtot * (double)nb;  // project_occ's denominator
    auto occ_shift = [&](double num) { return occ_den > 0.0 ? num / occ_den : 0.0; };

    std::vector<double> hist_e((size_t)std::max<int64_t>(max_iter, 1)), hist_g((size_t)std::max<int64_t>(max_iter, 1));
    int s = 0;
    double Delta = cfg->tr_delta0;
    int64_t k = 0;
    bool converged = false;
    const int64_t cg_max = cfg->tr_cg_max;
    while (k < max_iter) {
        const double grad_norm = hg[s];
        hist_e[k] = hE[s];
        hist_g[k] = grad_norm;
        if (grad_norm < tol_g) {
            converged = true;
            ++k;
            break;
        }
        if (Delta < 1e-10) break;  // solver_rtr.hpp:379 (Delta does not change before that test)
        const double lam = hlam[s];
        const double* ek = eps[s];
        const double* pk = p[s];
        const double* pen = defl ? &R->pen[s] : nullptr;
        const double2* hmat = static_cast<const double2*>(K->h);
        // one Hessian-vector product of direction mode `mode` (its sums land in R)
        auto hvp_step = [&](int mode, double beta, double rz_old) -> int {
            CPPHF_TRY(launch_direction(rX, rp, ek, pk, K->w2d, Q[s], vX, vp, dX, dp, dP, nk, nb, T_r, lam, beta, 0.0,
                                       rz_old, mode, R, st));
            CPPHF_TRY(build_fock(&Kr, dP, solver_sigma(&Kr, Sig), F, nullptr, nullptr, nullptr, fws, L.fock_bytes, st));
            return launch_hvp(dX, dp, Q[s], pk, Ft[s], F, hmat, dP, pen, K->w2d, HDX, HDp, nk, nb, T_r, R, st);
        };
        auto update = [&](int mode, double a, double shift_h) -> int {
            k_rtr_update<<<flat_blocks(nk * nb * nb, 256), 256, 0, st>>>(mode, a, shift_h, G[s], vX, HvX, rX, dX, HDX,
                                                                         vp, Hvp, rp, dp, HDp, ek, pk, K->w2d, nk, nb,
                                                                         T_r, lam, R);
            CPPHF_LAUNCH_CHECK("rtr cg update");
            return CPPHF_OK;
        };
        // ---- Steihaug truncated CG (solver_rtr.hpp:304-364) ----
        // r = -G, v = Hv = 0 and the first direction d = z(r) with its product
        // are queued together; every later step queues the next direction and
        // product behind the vector update before reading the sums of both
        // (one synchronisation per step).  A product queued for a step the host
        // then does not take only overwrote d, which the solve no longer needs.
        CPPHF_TRY(update(2, 0.0, 0.0));
        if (cg_max > 0) CPPHF_TRY(hvp_step(0, 0.0, 1.0));
        CPPHF_TRY(read_sums(kSumDD, kSumA4 + 1));
        double rz = sums[kSumA1] + sums[kSumA2] - occ_shift(sums[kSumA3]) * sums[kSumA4];
        for (int64_t cg = 0; cg < cg_max; ++cg) {
            const double shift_h = occ_shift(sums[kSumB4]);
            const double dHd = sums[kSumB1] + sums[kSumB2] - shift_h * sums[kSumB3];
            const double dd = sums[kSumDD], vd = sums[kSumVD], vv = sums[kSumVV];
            bool boundary = dHd <= 1e-14 * dd;  // negative curvature
            if (!boundary) {
                const double alpha = rz / dHd;
                const double s2 = vv + 2.0 * alpha * vd + alpha * alpha * dd;  // |v + alpha d|^2
                boundary = std::sqrt(std::max(0.0, s2)) >= Delta;
            }
            if (boundary) {  // to the positive root of |v + t d|^2 = Delta^2
                const double a = dd, b = 2.0 * vd, c = std::sqrt(std::max(0.0, vv));
                const double cc = c * c - Delta * Delta;
                const double tt = (-b + std::sqrt(std::max(b * b - 4.0 * a * cc, 0.0))) / (2.0 * a + 1e-30);
                CPPHF_TRY(update(1, tt, shift_h));
                break;
            }
            CPPHF_TRY(update(0, rz / dHd, shift_h));
            const bool more = cg + 1 < cg_max;
            if (more) CPPHF_TRY(hvp_step(3, 0.0, rz));
            CPPHF_TRY(read_sums(kSumDD, kSumA4 + 1));
            if (std::sqrt(std::max(0.0, sums[kSumRR])) < 0.05 * grad_norm || !more) break;
            const double shift_z = occ_shift(sums[kSumA3]);
            rz = sums[kSumA1] + sums[kSumA2] - shift_z * sums[kSumA4];
        }
        // ---- predicted reduction in energy units (solver_rtr.hpp:366-378), read with the trial state ----
        k_rtr_model<<<flat_blocks(nk * nb * nb, 256), 256, 0, st>>>(G[s], vX, HvX, vp, Hvp, K->w2d, nk, nb, R);
        CPPHF_LAUNCH_CHECK("rtr model");

        // ---- retraction Q <- Q Cayley(tau = -1, vX), trial mu and occupations ----
        const int t = s ^ 1;
        if (rtr_small_supported(nb)) {  // Cayley factor by elimination
            CPPHF_TRY(rtr_small_retract(vX, Q[s], Ft[s], Q[t], ew, nk, nb, st));
        } else {  // spectral Cayley factor (solver_rtr.hpp:386-387)
            CPPHF_TRY(eigh_batched(vX, lamd, Vd, nk, nb, 1, nullptr, st));
            CPPHF_TRY(launch_retract(Vd, lamd, Q[s], Ft[s], Q[t], ew, nk, nb, st));
        }
        CPPHF_TRY(mu_solve(ew, wn, nk, nb, n_t, &R->mu[s], T_r, mu_it, 1, &R->mu[t], mws, L.mu_bytes, st));
        CPPHF_TRY(occupy(t, ew));
        CPPHF_TRY(eval(t, true));  // the one Fock build at the trial point
        const double pred = -(sums[kSumGV] + 0.5 * (sums[kSumVHX] + sums[kSumVHP]));
        const double vnorm = std::sqrt(std::max(0.0, sums[kSumVVX] + sums[kSumVVP]));
        const double E = hE[s], E_t = hE[t], grad_t = hg[t];

        // ---- acceptance and trust radius (solver_rtr.hpp:398-420) ----
        const double noise = 1e-12 * std::max(std::fabs(E), 1.0);
        bool accept;
        if (pred <= noise) {
            accept = (grad_t <= grad_norm) && (E_t <= E + noise);
            if (!accept) Delta *= 0.5;
        } else {
            const double ratio = (E - E_t) / pred;
            if (ratio < 0.25)
                Delta *= 0.25;
            else if (ratio > 0.75 && vnorm > 0.9 * Delta)
                Delta = std::min(2.0 * Delta, 5.0);
            accept = ratio > 0.1;
        }
        if (accept) s = t;
        ++k;
    }

    // ---- finalize (solver_rtr.hpp:437-443) ----
    CPPHF_TRY(dm_density(Q[s], p[s], P, nk, nb, st));
    CPPHF_TRY(finish_density());
    CPPHF_TRY(build_fock(K, P, solver_sigma(K, Sig), F, nullptr, &R->efin, nullptr, fws, L.fock_bytes, st));
    if (Q_out) CPPHF_CUDA(cudaMemcpyAsync(Q_out, Q[s], fbytes, cudaMemcpyDeviceToDevice, st));
    if (p_out) CPPHF_CUDA(cudaMemcpyAsync(p_out, p[s], vbytes, cudaMemcpyDeviceToDevice, st));
    if (D_out) CPPHF_CUDA(cudaMemcpyAsync(D_out, P, fbytes, cudaMemcpyDeviceToDevice, st));
    if (F_out) CPPHF_CUDA(cudaMemcpyAsync(F_out, F, fbytes, cudaMemcpyDeviceToDevice, st));
    CPPHF_CUDA(cudaMemcpyAsync(hb, &R->efin, sizeof(double), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaMemcpyAsync(hb + 1, &R->mu[s], sizeof(double), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    res->energy = hb[0];
    res->mu = hb[1];
    res->n_iter = k;
    res->converged = converged ? 1 : 0;
    for (int64_t i = 0; i < k; ++i) {
        if (hist_E) hist_E[i] = hist_e[i];
        if (hist_G) hist_G[i] = hist_g[i];
    }
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

size_t cpphf_rtr_joint_hvp_workspace_bytes(const cpphf_kernel* K) {
    if (!K) return 0;
    const size_t fld = (sizeof(double2) * (size_t)K->nk1 * K->nk2 * K->nb * K->nb + 255) & ~(size_t)255;
    return 3 * fld + ((sizeof(cpphf::RtrScalars) + 255) & ~(size_t)255) + cpphf::fock_bytes_rtr(K);
}

int cpphf_rtr_joint_hvp(const cpphf_kernel* K, const void* X, const double* dp, const void* Q, const double* p,
                        const void* Ft, void* HX, double* Hp, void* workspace, size_t workspace_bytes, void* stream) {
    using namespace cpphf;
    CPPHF_TRY(validate_kernel(K));
    if (!X || !dp || !Q || !p || !Ft || !HX || !Hp) return fail(CPPHF_ERR_INVALID, "_rtr_joint_hvp: null argument");
    CPPHF_TRY(rtr_check_nb(K->nb));
    const size_t need = cpphf_rtr_joint_hvp_workspace_bytes(K);
    if (!workspace || workspace_bytes < need)
        return fail(CPPHF_ERR_INVALID, "_rtr_joint_hvp: workspace too small (" + std::to_string(need) +
                                           " bytes needed)");
    init_rtr_attrs();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nk = K->nk1 * K->nk2;
    const int nb = (int)K->nb;
    const size_t fld = (sizeof(double2) * (size_t)nk * nb * nb + 255) & ~(size_t)255;
    unsigned char* W = static_cast<unsigned char*>(workspace);
    double2* dP = reinterpret_cast<double2*>(W);
    double2* Sig = reinterpret_cast<double2*>(W + fld);
    double2* F = reinterpret_cast<double2*>(W + 2 * fld);
    const size_t a = 3 * fld;
    RtrScalars* R = reinterpret_cast<RtrScalars*>(W + a);
    void* fws = W + a + ((sizeof(RtrScalars) + 255) & ~(size_t)255);
    const size_t fb = fock_bytes_rtr(K);
    const double T_r = std::max(K->T, 1.0e-12);
    cpphf_kernel Kr = *K;
    Kr.has_refP = 0;
    CPPHF_CUDA(cudaMemsetAsync(R, 0, sizeof(RtrScalars), st));
    k_rtr_wsum<<<flat_blocks(nk, 256), 256, 0, st>>>(K->w2d, nk, R);
    CPPHF_LAUNCH_CHECK("rtr weight sum");
    // dP from the given direction (X, dp): mode 2 reads it unchanged
    CPPHF_TRY(launch_direction(nullptr, nullptr, nullptr, p, K->w2d, static_cast<const double2*>(Q), nullptr,
                               nullptr, const_cast<double2*>(static_cast<const double2*>(X)),
                               const_cast<double*>(dp), dP, nk, nb, T_r, 0.0, 0.0, 0.0, 1.0, 2, R, st));
    CPPHF_TRY(build_fock(&Kr, dP, solver_sigma(&Kr, Sig), F, nullptr, nullptr, nullptr, fws, fb, st));
    CPPHF_TRY(launch_hvp(static_cast<const double2*>(X), dp, static_cast<const double2*>(Q), p,
                         static_cast<const double2*>(Ft), F, static_cast<const double2*>(K->h), dP, nullptr, K->w2d,
                         static_cast<double2*>(HX), Hp, nk, nb, T_r, R, st));
    k_rtr_project_occ<<<flat_blocks(nk * nb, 256), 256, 0, st>>>(Hp, nk * nb, nb, R);
    CPPHF_LAUNCH_CHECK("rtr project_occ");
    return CPPHF_OK;
}

size_t cpphf_deflation_bias_workspace_bytes(int64_t n_deflation) {
    return ((sizeof(cpphf::RtrScalars) + 255) & ~(size_t)255) +
           sizeof(double) * (size_t)std::max<int64_t>(n_deflation, 1) + 4 * sizeof(double);
}

int cpphf_deflation_bias(const void* P, const void* targets, int64_t n_deflation, const double* w2d, int64_t nk1,
                         int64_t nk2, int64_t nb, double sigma, double length, void* S_pen, double* phi_diag,
                         void* workspace, size_t workspace_bytes, void* stream) {
    using namespace cpphf;
    if (!P || !w2d || !S_pen || !phi_diag) return fail(CPPHF_ERR_INVALID, "_deflation_bias: null argument");
    if (nk1 < 1 || nk2 < 1 || nb < 1 || n_deflation < 0) return fail(CPPHF_ERR_INVALID, "_deflation_bias: bad shape");
    if (n_deflation > kMaxDeflation) return fail(CPPHF_ERR_UNSUPPORTED, "more than 256 deflation targets");
    const size_t need = cpphf_deflation_bias_workspace_bytes(n_deflation);
    if (!workspace || workspace_bytes < need)
        return fail(CPPHF_ERR_INVALID, "_deflation_bias: workspace too small (" + std::to_string(need) +
                                           " bytes needed)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nk = nk1 * nk2;
    const size_t fbytes = sizeof(double2) * (size_t)nk * nb * nb;
    phi_diag[0] = 0.0;
    phi_diag[1] = 0.0;
    if (n_deflation == 0 || sigma == 0.0 || !targets) {
        CPPHF_CUDA(cudaMemsetAsync(S_pen, 0, fbytes, st));
        CPPHF_CUDA(cudaStreamSynchronize(st));
        return CPPHF_OK;
    }
    unsigned char* W = static_cast<unsigned char*>(workspace);
    RtrScalars* R = reinterpret_cast<RtrScalars*>(W);
    double* d2 = reinterpret_cast<double*>(W + ((sizeof(RtrScalars) + 255) & ~(size_t)255));
    double* out2 = d2 + std::max<int64_t>(n_deflation, 1);
    CPPHF_CUDA(cudaMemsetAsync(R, 0, sizeof(RtrScalars), st));
    CPPHF_TRY(deflation(static_cast<const double2*>(P), static_cast<const double2*>(targets), n_deflation, w2d, nk,
                        (int)nb, sigma, length, nullptr, static_cast<double2*>(S_pen), nullptr, out2, out2 + 1, d2, R,
                        st));
    CPPHF_CUDA(cudaMemcpyAsync(phi_diag, out2, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    return CPPHF_OK;
}

}  // extern "C"
