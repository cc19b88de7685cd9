// Register-resident FFT codelets and the four-step line transform used by the
// exchange passes for mesh axes of supported lengths.
//
// A line of N = N1 * N2 points (one channel) is spread over N2 threads for the
// first half and N1 threads for the second half:
//   forward, n = N2 n1 + n2, k = k1 + N1 k2:
//     thread n2: v[n1] = x[N2 n1 + n2]; DFT_N1 over n1; v[k1] *= W_N^{n2 k1}
//     (shared-memory transpose [N1][N2])
//     thread k1: u[n2] = Y[k1][n2]; DFT_N2 over n2 -> u[k2] = X[k1 + N1 k2]
//   inverse, starting from that distribution (thread k1 holds X[k1 + N1 k2]):
//     DFT^-1_N2 over k2 -> u[na]; u[na] *= W_N^{-na k1}
//     (shared-memory transpose)
//     thread na: v[k1] = Z[k1][na]; DFT^-1_N1 over k1 -> v[nb] = x[na + N2 nb]
// so the inverse lands on the same index set each thread loaded, and all
// arithmetic happens in registers with compile-time twiddles.  Codelets are
// built recursively by Cooley-Tukey from radix-2/3/4/5 kernels.
#pragma once

#include "common.cuh"

namespace cpphf {

// ---------------------------------------------------------------------------
// compile-time twiddles W_N^m = exp(-2 pi i m / N) (Taylor series on [0, pi/4]
// plus octant symmetry; accurate to a few ulp)
// ---------------------------------------------------------------------------
constexpr double kPiQ = 0.78539816339744830961566084581987572;  // pi / 4

constexpr double ct_sin_small(double x) {
    double x2 = x * x, t = x, s = x;
    for (int k = 1; k <= 12; ++k) {
        t *= -x2 / double((2 * k) * (2 * k + 1));
        s += t;
    }
    return s;
}
constexpr double ct_cos_small(double x) {
    double x2 = x * x, t = 1.0, s = 1.0;
    for (int k = 1; k <= 12; ++k) {
        t *= -x2 / double((2 * k - 1) * (2 * k));
        s += t;
    }
    return s;
}

template <int N>
struct TwTab {
    double re[N > 0 ? N : 1];
    double im[N > 0 ? N : 1];
    constexpr TwTab() : re(), im() {
        for (int m = 0; m < N; ++m) {
            const int q = 8 * m, o = q / N, r = q - o * N;
            double c = 0.0, s = 0.0;
            int k = 0;
            if (o % 2 == 0) {
                const double x = kPiQ * (double(r) / double(N));
                c = ct_cos_small(x);
                s = ct_sin_small(x);
                k = o / 2;
            } else {
                const double x = kPiQ - kPiQ * (double(r) / double(N));
                c = ct_sin_small(x);
                s = ct_cos_small(x);
                k = (o - 1) / 2;
            }
            for (int j = 0; j < k; ++j) {
                const double t = c;
                c = -s;
                s = t;
            }
            re[m] = c;
            im[m] = -s;
        }
    }
};

template <int N, bool INV, class C>
__device__ __forceinline__ C ctw(int m) {
    constexpr TwTab<N> T{};
    using R = decltype(C{}.x);
    return mk((R)T.re[m % N], (R)(INV ? -T.im[m % N] : T.im[m % N]));
}

// multiply by a compile-time twiddle, skipping trivial ones
template <int N, bool INV, class C>
__device__ __forceinline__ C twmul(C a, int m) {
    m %= N;
    if (m == 0) return a;
    if (4 * m == N) return INV ? mk(-a.y, a.x) : mk(a.y, -a.x);       // -+i
    if (2 * m == N) return mk(-a.x, -a.y);
    if (4 * m == 3 * N) return INV ? mk(a.y, -a.x) : mk(-a.y, a.x);
    return cmul(a, ctw<N, INV, C>(m));
}

constexpr int pick_radix(int n) {
    return (n % 4 == 0 && n != 8) ? 4 : (n % 2 == 0 ? 2 : (n % 3 == 0 ? 3 : (n % 5 == 0 ? 5 : n)));
}

template <int N, bool INV, class C>
__device__ __forceinline__ void dft(C (&x)[N]) {
    using R = decltype(C{}.x);
    constexpr int S = INV ? 1 : -1;
    if constexpr (N == 1) {
        return;
    } else if constexpr (N == 2) {
        const C a = x[0], b = x[1];
        x[0] = cadd(a, b);
        x[1] = csub(a, b);
    } else if constexpr (N == 3) {
        const R h = (R)0.86602540378443864676;
        const C a = x[0], t1 = cadd(x[1], x[2]), t2 = csub(x[1], x[2]);
        const C m = mk(a.x - (R)0.5 * t1.x, a.y - (R)0.5 * t1.y);
        const C r = cmuli<S>(cscale(t2, h));
        x[0] = cadd(a, t1);
        x[1] = cadd(m, r);
        x[2] = csub(m, r);
    } else if constexpr (N == 4) {
        const C a = x[0], b = x[1], c = x[2], d = x[3];
        const C s0 = cadd(a, c), d0 = csub(a, c), s1 = cadd(b, d), d1 = cmuli<S>(csub(b, d));
        x[0] = cadd(s0, s1);
        x[1] = cadd(d0, d1);
        x[2] = csub(s0, s1);
        x[3] = csub(d0, d1);
    } else if constexpr (N == 5) {
        C out[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            C acc = x[0];
#pragma unroll
            for (int i = 1; i < 5; ++i) acc = cadd(acc, twmul<5, INV>(x[i], i * m));
            out[m] = acc;
        }
#pragma unroll
        for (int m = 0; m < 5; ++m) x[m] = out[m];
    } else {
        constexpr int RR = pick_radix(N);
        constexpr int M = N / RR;
        static_assert(RR * M == N && RR < N, "unsupported codelet size");
        C sub[RR][M];
#pragma unroll
        for (int r = 0; r < RR; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) sub[r][m] = x[r + RR * m];
#pragma unroll
        for (int r = 0; r < RR; ++r) dft<M, INV>(sub[r]);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            C t[RR];
#pragma unroll
            for (int r = 0; r < RR; ++r) t[r] = twmul<N, INV>(sub[r][m], r * m);
            dft<RR, INV>(t);
#pragma unroll
            for (int q = 0; q < RR; ++q) x[m + M * q] = t[q];
        }
    }
}

// (N1, N2) split of the supported line lengths; {0, 0} = use the generic path.
struct Split {
    int n1, n2;
};
__host__ __device__ constexpr Split split_of(int n) {
    switch (n) {
        case 1: return {1, 1};
        case 2: return {2, 1};
        case 3: return {3, 1};
        case 4: return {4, 1};
        case 5: return {5, 1};
        case 6: return {3, 2};
        case 8: return {4, 2};
        case 9: return {3, 3};
        case 12: return {4, 3};
        case 16: return {4, 4};
        case 18: return {6, 3};
        case 24: return {6, 4};
        case 32: return {8, 4};
        case 36: return {6, 6};
        case 48: return {8, 6};
        case 64: return {8, 8};
        case 72: return {9, 8};
        case 96: return {12, 8};
        case 128: return {16, 8};
        case 144: return {12, 12};
        case 192: return {16, 12};
        case 256: return {16, 16};
        case 288: return {18, 16};
        default: return {0, 0};
    }
}

// Runtime twiddle table W_N^m in shared memory for the four-step inter-stage factors.
template <class C>
__device__ __forceinline__ void build_line_twiddles(C* tw, int n) {
    using R = decltype(C{}.x);
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        tw[m] = mk((R)c, (R)s);
    }
}

}  // namespace cpphf
