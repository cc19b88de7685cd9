// Tile helpers of the small-nb (2, 4, 6, 8) per-k kernels: a group of GS
// threads (nb rounded up to a power of two) owns one k-point, thread r owns row
// r of every matrix, and a CTA of kThreads threads stages KT = kThreads / GS
// k-points per tile through shared memory (coalesced loads and stores into a
// padded layout).  Used by the direct-minimisation (dm_small.cu) and
// trust-region Newton (rtr_small.cu) kernels.
#pragma once

#include "common.cuh"

#include <algorithm>

namespace cpphf {
namespace tile {

constexpr int kThreads = 128;

// Matrix stride in double2 units: >= nb * ld and, with 4 groups per warp
// (gs = 8), congruent to 2 or 6 mod 8 so the groups' broadcast reads use
// different banks; odd for smaller groups.
constexpr int pad_ms(int nb, int ld, int gs) {
    int m = nb * ld;
    if (gs == 8) {
        while (m % 8 != 2 && m % 8 != 6) ++m;
    } else if (m % 2 == 0) {
        ++m;
    }
    return m;
}

template <int NB>
struct Geo {
    static constexpr int GS = NB <= 2 ? 2 : (NB <= 4 ? 4 : 8);        // group size
    static constexpr int KT = kThreads / GS;                           // k-points per CTA tile
    static constexpr int NB2 = NB * NB;
    static constexpr int LD = NB + 1;                                  // padded row stride
    static constexpr int MS = pad_ms(NB, LD, GS);                      // padded matrix stride
    static constexpr int TILE = KT * MS;                               // shared double2 per staged tile
    static constexpr int PER = (KT * NB2 + kThreads - 1) / kThreads;  // elements per thread per tile
};

// coalesced global (dense k-blocks) -> shared (padded) copy of one tile; all
// loads are issued before the first shared store
template <int NB>
__device__ __forceinline__ void tile_load(double2* s, const double2* __restrict__ g, int nkt) {
    using G = Geo<NB>;
    const int n = nkt * G::NB2;
    double2 v[G::PER];
#pragma unroll
    for (int u = 0; u < G::PER; ++u) {
        const int e = threadIdx.x + u * kThreads;
        v[u] = (e < n) ? g[e] : mk(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < G::PER; ++u) {
        const int e = threadIdx.x + u * kThreads;
        if (e < n) {
            const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
            s[kl * G::MS + i * G::LD + j] = v[u];
        }
    }
}

// 16-byte asynchronous global -> shared copies (cp.async, L2 only) and their
// commit / wait: the loads of the next tile are issued before the current one
// is processed (the wait is on this thread's own copies; it cannot hang).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<unsigned>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// every group but the most recent one has landed
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// tile_load as asynchronous copies into the padded layout (committed by the caller)
template <int NB>
__device__ __forceinline__ void tile_load_async(double2* s, const double2* __restrict__ g, int nkt) {
    using G = Geo<NB>;
    const int n = nkt * G::NB2;
#pragma unroll
    for (int u = 0; u < G::PER; ++u) {
        const int e = threadIdx.x + u * kThreads;
        if (e < n) {
            const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
            cp_async16(&s[kl * G::MS + i * G::LD + j], g + e);
        }
    }
}

template <int NB>
__device__ __forceinline__ void tile_store(double2* g, const double2* s, int nkt) {
    using G = Geo<NB>;
    const int n = nkt * G::NB2;
#pragma unroll
    for (int u = 0; u < G::PER; ++u) {
        const int e = threadIdx.x + u * kThreads;
        if (e < n) {
            const int kl = e / G::NB2, rem = e - kl * G::NB2, i = rem / NB, j = rem - i * NB;
            g[e] = s[kl * G::MS + i * G::LD + j];
        }
    }
}

template <int NB>
__device__ __forceinline__ unsigned group_mask(int lane) {
    using G = Geo<NB>;
    const unsigned base = (1u << G::GS) - 1u;
    return G::GS == 32 ? 0xffffffffu : (base << ((lane / G::GS) * G::GS));
}


// ---------------------------------------------------------------------------
// Cayley unitary U(tau) = (I + tau d/2)^{-1} (I - tau d/2) of one k-point by
// Gauss-Jordan elimination, one row per thread (row r of the result in u[]).
// At step pp the owner of row pp publishes its row through the group's shared
// slot `piv` (two slots, used alternately, so one group barrier per step
// suffices); every thread then forms the reciprocal pivot itself, and the
// others subtract (f / pivot) times the published row, touching only the
// columns right of the pivot in the left block (the ones left of it are
// already zero).  The pivot rows are not normalised during the elimination:
// the owner's update is the same instruction stream with f = 0, so a group
// never diverges, and every row is divided by its own pivot (kept from its
// step) at the end.  `piv` holds 2 * 2 * NB values per group.
// With TR the elimination runs on the transposed system (thread r reads
// column r of d): U^T = (M^T)^{-1} N^T with M, N = I +- tau d/2 commuting,
// and M^T = I + (skew-Hermitian) as well, so u[] is column r of U.
// ---------------------------------------------------------------------------
// (row_cayley_reg takes this thread's row of d, or column with TR, in registers)
template <int NB>
__device__ __forceinline__ void row_cayley_reg(const double2 (&dv)[NB], double tau, int r, double2* piv,
                                               double2 (&u)[NB], unsigned mask) {
    double2 mrow[NB];
    const double h = 0.5 * tau;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const double2 a = cscale(dv[j], h);
        const double one = (j == r) ? 1.0 : 0.0;
        mrow[j] = mk(one + a.x, a.y);
        u[j] = mk(one - a.x, -a.y);
    }
    double2 rs = mk(1.0, 0.0);  // reciprocal of this row's pivot
#pragma unroll
    for (int pp = 0; pp < NB; ++pp) {
        double2* slot = piv + (pp & 1) * 2 * NB;
        if (r == pp) {
#pragma unroll
            for (int j = pp; j < NB; ++j) slot[j] = mrow[j];
#pragma unroll
            for (int j = 0; j < NB; ++j) slot[NB + j] = u[j];
        }
        __syncwarp(mask);
        const double2 pv = slot[pp];
        const double inv = 1.0 / (pv.x * pv.x + pv.y * pv.y);
        const double2 rp = mk(pv.x * inv, -pv.y * inv);
        const bool own = r == pp;
        if (own) rs = rp;
        const double2 f = own ? mk(0.0, 0.0) : cmul(mrow[pp], rp);
#pragma unroll
        for (int j = pp + 1; j < NB; ++j) mrow[j] = csub(mrow[j], cmul(f, slot[j]));
#pragma unroll
        for (int j = 0; j < NB; ++j) u[j] = csub(u[j], cmul(f, slot[NB + j]));
    }
#pragma unroll
    for (int j = 0; j < NB; ++j) u[j] = cmul(u[j], rs);
    __syncwarp(mask);  // the last step's readers are done before `piv` is reused
}

template <int NB, int LD, bool TR = false>
__device__ __forceinline__ void row_cayley(const double2* d, double tau, int r, double2* piv, double2 (&u)[NB],
                                           unsigned mask) {
    double2 dv[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) dv[j] = TR ? d[j * LD + r] : d[r * LD + j];
    row_cayley_reg<NB>(dv, tau, r, piv, u, mask);
}

// Two Cayley factors U(tau_a), U(tau_b) of the same d in lockstep: one pivot
// publication (both rows) and one group barrier per step for both
// eliminations, so their dependent FP64 chains interleave.  With M = I + tau d/2,
// U = M^{-1} (I - tau d/2) = 2 M^{-1} - I: the elimination runs on [M | I],
// whose right-hand block has filled in only columns 0..pp when pivot pp is
// eliminated, so each step updates pp + 1 right-hand columns instead of nb.
// As in row_cayley the pivot rows stay unnormalised (no divergence in the
// group) and each row is divided by its pivot at the end; with TR the results
// are columns of U (U^T = 2 (M^T)^{-1} - I).
// M = I + (skew-Hermitian) is well conditioned and the elimination needs no
// pivoting.  `piv` holds 2 * 4 * NB values per group.
template <int NB>
__device__ __forceinline__ void row_cayley2_reg(const double2 (&dv)[NB], double tau_a, double tau_b, int r,
                                                double2* piv, double2 (&ua)[NB], double2 (&ub)[NB], unsigned mask) {
    double2 ma[NB], mb[NB];
    const double ha = 0.5 * tau_a, hb = 0.5 * tau_b;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const double2 a = cscale(dv[j], ha), b = cscale(dv[j], hb);
        const double one = (j == r) ? 1.0 : 0.0;
        ma[j] = mk(one + a.x, a.y);
        mb[j] = mk(one + b.x, b.y);
        ua[j] = mk(one, 0.0);  // right-hand block: row r of I, then of M^{-1} times the pivot
        ub[j] = mk(one, 0.0);
    }
    double2 rsa = mk(1.0, 0.0), rsb = mk(1.0, 0.0);  // reciprocals of this row's pivots
#pragma unroll
    for (int pp = 0; pp < NB; ++pp) {
        double2* slot = piv + (pp & 1) * 4 * NB;
        if (r == pp) {
#pragma unroll
            for (int j = pp; j < NB; ++j) {
                slot[j] = ma[j];
                slot[2 * NB + j] = mb[j];
            }
#pragma unroll
            for (int j = 0; j <= pp; ++j) {
                slot[NB + j] = ua[j];
                slot[3 * NB + j] = ub[j];
            }
        }
        __syncwarp(mask);
        const double2 pa = slot[pp], pb = slot[2 * NB + pp];
        const double ia = 1.0 / (pa.x * pa.x + pa.y * pa.y);
        const double ib = 1.0 / (pb.x * pb.x + pb.y * pb.y);
        const double2 ra = mk(pa.x * ia, -pa.y * ia), rb = mk(pb.x * ib, -pb.y * ib);
        const bool own = r == pp;
        if (own) {
            rsa = ra;
            rsb = rb;
        }
        const double2 fa = own ? mk(0.0, 0.0) : cmul(ma[pp], ra);
        const double2 fb = own ? mk(0.0, 0.0) : cmul(mb[pp], rb);
#pragma unroll
        for (int j = pp + 1; j < NB; ++j) {
            ma[j] = csub(ma[j], cmul(fa, slot[j]));
            mb[j] = csub(mb[j], cmul(fb, slot[2 * NB + j]));
        }
#pragma unroll
        for (int j = 0; j <= pp; ++j) {
            ua[j] = csub(ua[j], cmul(fa, slot[NB + j]));
            ub[j] = csub(ub[j], cmul(fb, slot[3 * NB + j]));
        }
    }
    // U = 2 M^{-1} - I, row r of M^{-1} being the right-hand row over its pivot
    rsa = mk(2.0 * rsa.x, 2.0 * rsa.y);
    rsb = mk(2.0 * rsb.x, 2.0 * rsb.y);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const double one = (j == r) ? 1.0 : 0.0;
        const double2 a = cmul(ua[j], rsa), b = cmul(ub[j], rsb);
        ua[j] = mk(a.x - one, a.y);
        ub[j] = mk(b.x - one, b.y);
    }
    __syncwarp(mask);  // the last step's readers are done before `piv` is reused
}

template <int NB, int LD, bool TR = false>
__device__ __forceinline__ void row_cayley2(const double2* d, double tau_a, double tau_b, int r, double2* piv,
                                            double2 (&ua)[NB], double2 (&ub)[NB], unsigned mask) {
    double2 dv[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) dv[j] = TR ? d[j * LD + r] : d[r * LD + j];
    row_cayley2_reg<NB>(dv, tau_a, tau_b, r, piv, ua, ub, mask);
}

// diag(U^H Ft U) of one or two factors when thread r holds column r of each
// (ua, ub): diag_r = sum_j Re[conj(U_jr) (Ft U)_jr], Ft read row by row from
// the group's padded tile `sf` (one read serves both factors; no shuffles).
template <int NB, int LD, bool TWO>
__device__ __forceinline__ void col_diag_uhfu(const double2* sf, const double2 (&ua)[NB], const double2 (&ub)[NB],
                                              double& da, double& db) {
    double sa = 0.0, sb = 0.0;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        double2 ya = mk(0.0, 0.0), yb = mk(0.0, 0.0);
#pragma unroll
        for (int l = 0; l < NB; ++l) {
            const double2 f = sf[j * LD + l];
            cfma(ya, f, ua[l]);
            if (TWO) cfma(yb, f, ub[l]);
        }
        sa += ua[j].x * ya.x + ua[j].y * ya.y;
        if (TWO) sb += ub[j].x * yb.x + ub[j].y * yb.y;
    }
    da = sa;
    db = sb;
}

// diag(U^H Ft U) for the group: thread j holds Ft row j (ftj); it forms
// c_jq = conj(U_jq) (Ft U)_jq for every q from the group's padded U in shared
// memory `su`, and the group sums c_jq over j with xor-shuffles (fixed tree).
// Thread r returns diag_r.
template <int NB, int GS, int LD>
__device__ __forceinline__ double row_diag_uhfu(const double2 (&ftj)[NB], const double2* su, int r, unsigned mask,
                                                bool live) {
    double c[NB];
    const int rr = live ? r : 0;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        double2 wjq = mk(0.0, 0.0);
#pragma unroll
        for (int l = 0; l < NB; ++l) cfma(wjq, ftj[l], su[l * LD + q]);
        const double2 ujq = su[rr * LD + q];
        c[q] = live ? (ujq.x * wjq.x + ujq.y * wjq.y) : 0.0;
    }
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < NB; ++q) c[q] += __shfl_xor_sync(mask, c[q], o);
    double out = 0.0;
#pragma unroll
    for (int q = 0; q < NB; ++q)
        if (q == r) out = c[q];
    return out;
}


inline unsigned tiles_grid(int64_t nk, int KT, int cap) {
    const int64_t nt = (nk + KT - 1) / KT;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(nt, cap));
}


#define SMALL_DISPATCH(nb, X) \
    switch (nb) {             \
        case 2: X(2); break;  \
        case 4: X(4); break;  \
        case 6: X(6); break;  \
        case 8: X(8); break;  \
        default: return fail(CPPHF_ERR_UNSUPPORTED, "small-nb kernel called with unsupported nb"); \
    }


}  // namespace tile
}  // namespace cpphf
