// Per-k "team" helpers for batched small dense complex linear algebra.
//
// A team owns one k-point's nb x nb matrices in shared memory (row stride
// ld = nb + 1).  For nb <= 16 the team is one warp and a CTA runs
// kWarpTeams teams; for larger nb the team is the whole CTA.  Every kernel
// loops over k with a grid stride in units of teams, so warp teams never need
// a CTA-wide barrier inside the loop.
#pragma once

#include "common.cuh"

namespace cpphf {

constexpr int kTeamWarpMaxNb = 16;
constexpr int kWarpTeams = 4;
constexpr int kCtaTeamThreadsDense = 256;

template <bool WARP>
struct Team {
    int tid, nt, team, nteams;
    __device__ __forceinline__ Team() {
        if (WARP) {
            tid = threadIdx.x & 31;
            nt = 32;
            team = threadIdx.x >> 5;
            nteams = blockDim.x >> 5;
        } else {
            tid = threadIdx.x;
            nt = blockDim.x;
            team = 0;
            nteams = 1;
        }
    }
    __device__ __forceinline__ void sync() const {
        if (WARP)
            __syncwarp();
        else
            __syncthreads();
    }
};

__host__ __device__ __forceinline__ size_t team_mat_elems(int nb) { return (size_t)nb * (nb + 1); }

// dynamic shared memory of a team kernel: nmat team matrices + extra doubles
// per team, plus 64 doubles of block-reduction scratch
template <bool WARP>
inline size_t team_smem(int nb, int nmat, int extra_doubles_per_team) {
    const int teams = WARP ? kWarpTeams : 1;
    const size_t per = (sizeof(double2) * team_mat_elems(nb) * nmat + sizeof(double) * extra_doubles_per_team + 15) &
                       ~(size_t)15;
    return per * teams + sizeof(double) * 64;
}

template <bool WARP>
__device__ __forceinline__ double2* team_mats(unsigned char* raw, int nb, int nmat, int extra, int team) {
    const size_t per = (sizeof(double2) * team_mat_elems(nb) * nmat + sizeof(double) * extra + 15) & ~(size_t)15;
    return reinterpret_cast<double2*>(raw + per * team);
}

struct TeamLaunch {
    bool warp;
    int threads;
    unsigned grid;
};

// grid-stride launch over nk k-points in teams; the grid is capped so that the
// last-block reductions fit kTeamMaxPartials partials
constexpr int kTeamMaxPartials = 1024;

inline TeamLaunch team_launch(int64_t nk, int nb) {
    TeamLaunch L;
    L.warp = nb <= kTeamWarpMaxNb;
    L.threads = L.warp ? 32 * kWarpTeams : kCtaTeamThreadsDense;
    const int64_t teams = L.warp ? kWarpTeams : 1;
    const int64_t want = (nk + teams - 1) / teams;
    const int64_t cap = (int64_t)num_sms() * 16;
    L.grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
    return L;
}

inline unsigned flat_grid(int64_t n, int threads) {
    const int64_t want = (n + threads - 1) / threads;
    int64_t cap = (int64_t)num_sms() * 4;
    if (cap > kTeamMaxPartials) cap = kTeamMaxPartials;
    return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

#define TEAM_DISPATCH(L, kern, nmat, extra, ...)                                                  \
    do {                                                                                          \
        if (L.warp)                                                                               \
            kern<true><<<L.grid, L.threads, team_smem<true>(nb, nmat, extra), st>>>(__VA_ARGS__);  \
        else                                                                                      \
            kern<false><<<L.grid, L.threads, team_smem<false>(nb, nmat, extra), st>>>(__VA_ARGS__); \
        CPPHF_LAUNCH_CHECK(#kern);                                                                \
    } while (0)

template <bool WARP>
__device__ __forceinline__ void tload(double2* S, const double2* __restrict__ G, int nb, const Team<WARP>& t) {
    const int ld = nb + 1;
    for (int e = t.tid; e < nb * nb; e += t.nt) {
        const int i = e / nb, j = e - i * nb;
        S[i * ld + j] = G[e];
    }
}

template <bool WARP>
__device__ __forceinline__ void tstore(double2* G, const double2* S, int nb, const Team<WARP>& t) {
    const int ld = nb + 1;
    for (int e = t.tid; e < nb * nb; e += t.nt) {
        const int i = e / nb, j = e - i * nb;
        G[e] = S[i * ld + j];
    }
}

// C = op(A) op(B); op = conjugate transpose when AH / BH.  C must not alias A or B.
template <bool AH, bool BH, bool WARP>
__device__ __forceinline__ void tmm(double2* C, const double2* A, const double2* B, int nb,
                                    const Team<WARP>& t) {
    const int ld = nb + 1;
    for (int e = t.tid; e < nb * nb; e += t.nt) {
        const int i = e / nb, j = e - i * nb;
        double2 acc = mk(0.0, 0.0);
        for (int l = 0; l < nb; ++l) {
            const double2 a = AH ? cconj(A[l * ld + i]) : A[i * ld + l];
            const double2 b = BH ? cconj(B[j * ld + l]) : B[l * ld + j];
            cfma(acc, a, b);
        }
        C[i * ld + j] = acc;
    }
}

// Cayley factor c(tau, lam) = (1 + i tau lam / 2) / (1 - i tau lam / 2)
// (solver_dm.hpp:251-255): (1 - a^2 + 2 i a) / (1 + a^2), a = tau lam / 2.
__device__ __forceinline__ double2 cayley_factor(double lam, double tau) {
    const double a = 0.5 * tau * lam;
    // complex division (1 + i a) / (1 - i a)
    const double den = 1.0 + a * a;
    return mk((1.0 - a * a) / den, (2.0 * a) / den);
}

// Last-block-done reduction: every block adds NV values; the last block to
// arrive sums all partials (thread-strided, then a fixed tree: deterministic for
// a given grid) into out[0..NV) and
// resets the counter.  Returns true in every thread of the last block.
template <int NV, int M>
__device__ __forceinline__ bool reduce_last_block(double (&v)[NV], double* partials, unsigned* counter,
                                                  double* out, double (&red)[M]) {
    block_sum<NV>(v, red);
    __shared__ int is_last;
    const int G = gridDim.x;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) partials[(size_t)i * G + blockIdx.x] = v[i];
        __threadfence();
        const unsigned arrived = atomicAdd(counter, 1u);
        is_last = (arrived == (unsigned)G - 1) ? 1 : 0;
    }
    __syncthreads();
    if (is_last) {
        // whole last block: thread-strided partial sums, then the fixed block tree
        __threadfence();
        double acc[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = 0.0;
            for (int b = threadIdx.x; b < G; b += blockDim.x) s += __ldcg(&partials[(size_t)i * G + b]);
            acc[i] = s;
        }
        block_sum<NV>(acc, red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int i = 0; i < NV; ++i) out[i] = acc[i];
            atomicExch(counter, 0u);
        }
        __syncthreads();
    }
    return is_last != 0;
}

}  // namespace cpphf
