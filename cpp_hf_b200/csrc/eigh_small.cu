// Batched Hermitian eigendecomposition for small matrices (nb <= 8):
// Householder reduction to real tridiagonal form followed by implicit QL
// iterations, GS = (nb rounded up to 2, 4 or 8) lanes per matrix, everything in
// registers (replaces Eigen's SelfAdjointEigenSolver in cpp_hf linalg.hpp:39-66,
// which takes the same tridiagonal + QL route).
//
// Lane r of a group owns column r of A and row r of the accumulated unitary Z.
//  1. Reduction, k = 0 .. nb-3: lane k forms the reflector H = I - beta u u^H
//     that maps A[k+1:, k] to alpha e1 (alpha = -phase(x0) |x|, so the pivot
//     has no cancellation), broadcasts u; every lane j then forms
//     p_j = beta (A u)_j = beta A[:, j]^H u (A is Hermitian), the group sums
//     K = beta/2 u^H p, and with w = p - K u the similarity A <- H A H is the
//     rank-2 update A -= u w^H + w u^H (column j needs w: broadcast).  Z <- Z H
//     is a row-local update.
//  2. A unitary diagonal D (delta_0 = 1, delta_{k+1} = delta_k e_k/|e_k|) makes
//     the tridiagonal real: T' = D^H T D, Z <- Z D.
//  3. Implicit QL with Wilkinson shifts on (d, |e|) (Golub & Van Loan,
//     Matrix Computations, sec. 8.3; the tqli formulation of Press et al.):
//     every lane runs the same scalar recurrence and applies each Givens
//     rotation to its own row of Z.  The matrix is first scaled by a power of
//     two (exact) so that each rotation can use one reciprocal square root.
//  4. Stable ascending sort of the eigenvalues, columns of Z permuted to match.
// Loops over matrix indices are unrolled with compile-time indices so the
// per-lane arrays stay in registers.
#include "common.cuh"
#include "eigh.cuh"

#include <cstdlib>

namespace cpphf {

namespace {

constexpr int kHqlThreads = 128;
constexpr int kQlMaxIter = 60;  // QL iterations per eigenvalue before giving up

template <int NB>
struct HqlGeo {
    static constexpr int GS = NB <= 2 ? 2 : (NB <= 4 ? 4 : 8);
};

template <int GS>
__device__ __forceinline__ double group_sum(double v, unsigned mask) {
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

__device__ __forceinline__ double2 shfl2(double2 v, int src, unsigned mask) {
    return mk(__shfl_sync(mask, v.x, src), __shfl_sync(mask, v.y, src));
}

// four CTAs per SM (<= 128 registers, a few spilled): on the Fock matrices of
// an SCF solve (192 x 192, nb = 8) 194 us per call against 220 us at three CTAs
// without spills (on random Hermitian matrices three CTAs are 4 % faster).
// Splitting the kernel after the reduction (a QL kernel at 96 registers and
// five CTAs per SM, the tridiagonal and Z handed over through V) was slower:
// the QL is bound by its instruction count more than by latency.
template <int NB>
__global__ void __launch_bounds__(kHqlThreads, 4) k_eigh_hql(const double2* __restrict__ M, double* __restrict__ w,
                                                          double2* __restrict__ Vout, int64_t batch, int mode) {
    constexpr int GS = HqlGeo<NB>::GS;
    const int lane = threadIdx.x & 31;
    const int r = lane % GS;
    const int base = lane - r;
    const unsigned mask = (GS == 32 ? 0xffffffffu : (((1u << GS) - 1u) << base));
    const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / GS;
    if (k >= batch) return;  // whole group
    const double2* Mk = M + (size_t)k * NB * NB;

    // column r of herm(M) (mode 0) or herm(i M) (mode 1); lanes r >= NB hold zeros
    double2 a[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        double2 h = mk(0.0, 0.0);
        if (r < NB) {
            double2 x = Mk[i * NB + r], y = Mk[r * NB + i];
            if (mode == 1) {
                x = mk(-x.y, x.x);
                y = mk(-y.y, y.x);
            }
            h = mk(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
            if (i == r) h.y = 0.0;
        }
        a[i] = h;
    }
    // scale by a power of two so the largest entry is O(1): exact, and keeps the
    // QL rotations free of overflow; eigenvalues are scaled back at the end
    double amax = 0.0;
#pragma unroll
    for (int i = 0; i < NB; ++i) amax = fmax(amax, fmax(fabs(a[i].x), fabs(a[i].y)));
#pragma unroll
    for (int o = GS / 2; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(mask, amax, o));
    int ex = 0;
    if (amax > 0.0 && isfinite(amax)) frexp(amax, &ex);
#pragma unroll
    for (int i = 0; i < NB; ++i) a[i] = mk(ldexp(a[i].x, -ex), ldexp(a[i].y, -ex));
    double2 z[NB];  // row r of Z
#pragma unroll
    for (int j = 0; j < NB; ++j) z[j] = mk(j == r ? 1.0 : 0.0, 0.0);

    // ---- 1. Householder reduction ----
#pragma unroll
    for (int kk = 0; kk + 2 < NB; ++kk) {
        // lane kk: reflector of x = A[kk+1:, kk]
        double2 ul[NB];
        double bl = 0.0;
        double2 al = mk(0.0, 0.0);
        if (r == kk) {
            double xn2 = 0.0;
#pragma unroll
            for (int i = kk + 1; i < NB; ++i) xn2 += a[i].x * a[i].x + a[i].y * a[i].y;
            const double2 x0 = a[kk + 1];
            // entries are O(1) after the scaling, so the plain modulus cannot overflow
            const double ax0 = sqrt(fma(x0.x, x0.x, x0.y * x0.y));
            const double xn = sqrt(xn2);
#pragma unroll
            for (int i = 0; i < NB; ++i) ul[i] = mk(0.0, 0.0);
            if (xn > 0.0) {
                const double iax = ax0 > 0.0 ? 1.0 / ax0 : 0.0;
                const double2 ph = ax0 > 0.0 ? mk(x0.x * iax, x0.y * iax) : mk(1.0, 0.0);
                al = mk(-ph.x * xn, -ph.y * xn);
                ul[kk + 1] = mk(x0.x + ph.x * xn, x0.y + ph.y * xn);
#pragma unroll
                for (int i = kk + 2; i < NB; ++i) ul[i] = a[i];
                bl = 1.0 / (xn * (xn + ax0));
            } else {
                al = x0;
            }
        }
        double2 u[NB];
#pragma unroll
        for (int i = 0; i < NB; ++i) u[i] = (i > kk) ? shfl2(ul[i], base + kk, mask) : mk(0.0, 0.0);
        const double beta = __shfl_sync(mask, bl, base + kk);
        const double2 alpha = shfl2(al, base + kk, mask);
        if (beta != 0.0) {  // group-uniform
            // p_r = beta A[:, r]^H u
            double2 pr = mk(0.0, 0.0);
#pragma unroll
            for (int i = kk + 1; i < NB; ++i) cfma(pr, cconj(a[i]), u[i]);
            pr = cscale(pr, beta);
            // K = beta/2 sum_j conj(u_j) p_j (real for Hermitian A)
            double2 ur = u[0];
#pragma unroll
            for (int i = 1; i < NB; ++i)
                if (i == r) ur = u[i];
            if (r >= NB) ur = mk(0.0, 0.0);
            const double Kp = group_sum<GS>(ur.x * pr.x + ur.y * pr.y, mask);
            const double K = 0.5 * beta * Kp;
            const double2 wr = mk(pr.x - K * ur.x, pr.y - K * ur.y);
            double2 wv[NB];
#pragma unroll
            for (int i = 0; i < NB; ++i) wv[i] = shfl2(wr, base + i, mask);
            // column r: a -= u conj(w_r) + w conj(u_r)
            const double2 cw = cconj(wr), cu = cconj(ur);
#pragma unroll
            for (int i = kk + 1; i < NB; ++i) {
                a[i] = csub(a[i], cmul(u[i], cw));
                a[i] = csub(a[i], cmul(wv[i], cu));
            }
            // row r of Z: z <- z - beta (z . u) u^H
            double2 t = mk(0.0, 0.0);
#pragma unroll
            for (int j = kk + 1; j < NB; ++j) cfma(t, z[j], u[j]);
            t = cscale(t, beta);
#pragma unroll
            for (int j = kk + 1; j < NB; ++j) z[j] = csub(z[j], cmul(t, cconj(u[j])));
        }
        // exact tridiagonal shape of column / row kk
        if (r == kk) {
            a[kk + 1] = alpha;
#pragma unroll
            for (int i = kk + 2; i < NB; ++i) a[i] = mk(0.0, 0.0);
        } else if (r == kk + 1) {
            a[kk] = cconj(alpha);
        } else if (r > kk + 1) {
            a[kk] = mk(0.0, 0.0);
        }
    }

    // ---- 2. real tridiagonal ----
    double d[NB], e[NB];
    double2 sub[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        double2 di = a[0];
#pragma unroll
        for (int j = 1; j < NB; ++j)
            if (j == i) di = a[j];
        d[i] = __shfl_sync(mask, di.x, base + i);  // A_ii from lane i
        double2 si = mk(0.0, 0.0);
        if (i + 1 < NB) {
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j == i + 1) si = a[j];
            si = shfl2(si, base + i, mask);  // A_{i+1,i} from lane i
        }
        sub[i] = si;
    }
    double2 delta = mk(1.0, 0.0);
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        z[i] = cmul(z[i], delta);
        if (i + 1 < NB) {
            const double m = sqrt(fma(sub[i].x, sub[i].x, sub[i].y * sub[i].y));
            e[i] = m;
            if (m > 0.0) {
                const double im = 1.0 / m;
                delta = cmul(delta, mk(sub[i].x * im, sub[i].y * im));
            }
        } else {
            e[i] = 0.0;
        }
    }

    // ---- 3. implicit QL ----
    constexpr double kEps = 2.220446049250313e-16;
    // l unrolled: the sweeps for eigenvalue l address d, e and z at
    // compile-time offsets and issue only the rotations of rows l..NB-2
#pragma unroll
    for (int l = 0; l < NB; ++l) {
        int iter = 0;
        while (true) {
            // first m >= l with a negligible e[m] (m = NB-1 if none)
            int m = NB - 1;
#pragma unroll
            for (int i = NB - 2; i >= 0; --i) {
                if (i >= l) {
                    const double dd = fabs(d[i]) + fabs(d[i + 1]);
                    if (fabs(e[i]) <= kEps * dd) m = i;
                }
            }
            if (m == l || ++iter > kQlMaxIter) break;
            double dl = d[0], dl1 = d[0], el = e[0], dm = d[0];
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (j == l) {
                    dl = d[j];
                    el = e[j];
                }
                if (j == l + 1) dl1 = d[j];
                if (j == m) dm = d[j];
            }
            // Wilkinson shift: with t = d[l+1] - d[l], u = 2 e[l] and g0 = t / u,
            // el / (g0 + sign(g0) sqrt(g0^2 + 1)) = el u / (t + sign(t) sqrt(t^2 + u^2)):
            // one division instead of two (the tridiagonal is O(1), so t^2 + u^2
            // can only vanish by underflow; the two-division form covers that case)
            const double t = dl1 - dl, u2 = 2.0 * el;
            const double den = t + copysign(sqrt(fma(t, t, u2 * u2)), t);
            double g;
            if (den != 0.0) {
                g = dm - dl + el * u2 / den;
            } else {
                g = t / u2;
                g = dm - dl + el / (g + copysign(sqrt(fma(g, g, 1.0)), g));
            }
            double rr;
            double s = 1.0, c = 1.0, p = 0.0;
            bool under = false;
#pragma unroll
            for (int i = NB - 2; i >= 0; --i) {
                if (i >= l && i < m && !under) {
                    const double f = s * e[i], b = c * e[i];
                    // Givens pair from one reciprocal square root (the matrix was
                    // scaled to unit size, so f^2 + g^2 cannot overflow)
                    const double q = fma(f, f, g * g);
                    if (q == 0.0) {
                        e[i + 1] = 0.0;
                        d[i + 1] -= p;
                        under = true;
                    } else {
                        const double rinv = rsqrt(q);
                        rr = q * rinv;
                        e[i + 1] = rr;
                        s = f * rinv;
                        c = g * rinv;
                        g = d[i + 1] - p;
                        const double t = (d[i] - g) * s + 2.0 * c * b;
                        p = s * t;
                        d[i + 1] = g + p;
                        g = c * t - b;
                        const double2 zi = z[i], zi1 = z[i + 1];
                        z[i + 1] = mk(s * zi.x + c * zi1.x, s * zi.y + c * zi1.y);
                        z[i] = mk(c * zi.x - s * zi1.x, c * zi.y - s * zi1.y);
                    }
                }
            }
            if (under) {
#pragma unroll
                for (int j = 0; j < NB; ++j)
                    if (j == m) e[j] = 0.0;
                continue;
            }
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                if (j == l) {
                    d[j] -= p;
                    e[j] = g;
                }
                if (j == m) e[j] = 0.0;
            }
        }
    }

    // ---- 4. stable ascending order ----
    int rank[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        int rk = 0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
            if (d[j] < d[i] || (d[j] == d[i] && j < i)) ++rk;
        rank[i] = rk;
    }
    if (r < NB) {
        double2* Vrow = Vout + ((size_t)k * NB + r) * NB;
        double2 out[NB];
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            double2 v = z[0];
#pragma unroll
            for (int i = 0; i < NB; ++i)
                if (rank[i] == j) v = z[i];
            out[j] = v;
        }
#pragma unroll
        for (int j = 0; j < NB; ++j) Vrow[j] = out[j];
        if (r == 0) {
            double* wk = w + (size_t)k * NB;
#pragma unroll
            for (int i = 0; i < NB; ++i) {
                double v = d[0];
#pragma unroll
                for (int j = 0; j < NB; ++j)
                    if (rank[j] == i) v = d[j];
                wk[i] = ldexp(v, ex);
            }
        }
    }
}

}  // namespace

bool eigh_small_enabled(int64_t nb) { return nb >= 2 && nb <= 8; }

int eigh_small(const double2* M, double* w, double2* V, int64_t batch, int64_t nb, int mode, cudaStream_t st) {
    const int64_t threads = batch * (nb <= 2 ? 2 : (nb <= 4 ? 4 : 8));
    const unsigned grid = (unsigned)((threads + kHqlThreads - 1) / kHqlThreads);
    switch (nb) {
        case 2: k_eigh_hql<2><<<grid, kHqlThreads, 0, st>>>(M, w, V, batch, mode); break;
        case 3: k_eigh_hql<3><<<grid, kHqlThreads, 0, st>>>(M, w, V, batch, mode); break;
        case 4: k_eigh_hql<4><<<grid, kHqlThreads, 0, st>>>(M, w, V, batch, mode); break;
        case 5: k_eigh_hql<5><<<grid, kHqlThreads, 0, st>>>(M, w, V, batch, mode); break;
        case 6: k_eigh_hql<6><<<grid, kHqlThreads, 0, st>>>(M, w, V, batch, mode); break;
        case 7: k_eigh_hql<7><<<grid, kHqlThreads, 0, st>>>(M, w, V, batch, mode); break;
        case 8: k_eigh_hql<8><<<grid, kHqlThreads, 0, st>>>(M, w, V, batch, mode); break;
        default: return fail(CPPHF_ERR_UNSUPPORTED, "eigh_small: nb out of range");
    }
    CPPHF_LAUNCH_CHECK("eigh (Householder + QL)");
    return CPPHF_OK;
}

}  // namespace cpphf
