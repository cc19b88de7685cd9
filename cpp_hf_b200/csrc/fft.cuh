// Generic shared-memory batched 1-D FFT on a tile of n points x CB channels,
// for line lengths that have no register codelet (fft_reg.cuh).
//
// The tile is row-major [n][CB] complex in shared memory (channel fastest).  A
// plan is a list of radices whose product is n; every stage is an out-of-place
// Stockham step between two tile buffers
//
//   for butterfly j in [0, n/R), channel c, output m < R:
//       k = j mod Ns
//       y[(j/Ns) Ns R + k + m Ns] = sum_i x[j + i n/R] W_n^{i k n/(Ns R)} W_R^{i m}
//   Ns *= R
//
// computed one output per thread iteration directly from shared memory (no
// register arrays).  Twiddles come from one table W_n^m = exp(-2 pi i m / n)
// built per block with sincospi().
#pragma once

#include "common.cuh"

namespace cpphf {

constexpr int kMaxStages = 24;

struct FftPlan1D {
    int n;
    int nstages;
    int generic;  // unused by the generic path (kept for layout stability)
    int radix[kMaxStages];
};

// Host: factor n into stage radices (8s and 4s for powers of two, then 3, 5, 7,
// then remaining primes as generic stages).
inline bool make_plan(int n, FftPlan1D& pl) {
    pl.n = n;
    pl.nstages = 0;
    pl.generic = 0;
    if (n < 1) return false;
    int m = n, a = 0;
    while (m % 2 == 0) { m /= 2; ++a; }
    auto push = [&](int r) {
        if (pl.nstages >= kMaxStages) return false;
        pl.radix[pl.nstages++] = r;
        return true;
    };
    // powers of two: prefer 8, finish with 4 or 4*4 rather than 2 where possible
    if (a % 3 == 1 && a >= 4) {
        for (int i = 0; i < (a - 4) / 3; ++i) if (!push(8)) return false;
        if (!push(4) || !push(4)) return false;
    } else {
        for (int i = 0; i < a / 3; ++i) if (!push(8)) return false;
        if (a % 3 == 2) { if (!push(4)) return false; }
        if (a % 3 == 1) { if (!push(2)) return false; }
    }
    for (int p : {3, 5, 7}) {
        while (m % p == 0) { m /= p; if (!push(p)) return false; }
    }
    for (int p = 11; m > 1; p += 2) {
        while (m % p == 0) {
            m /= p;
            if (!push(p)) return false;
            pl.generic = 1;
        }
        if (p * p > m && m > 1) {  // m is prime
            if (!push(m)) return false;
            pl.generic = 1;
            m = 1;
        }
    }
    return true;
}

// W_n^m table (forward sign) in shared memory.
template <class C>
__device__ __forceinline__ void build_twiddles(C* tw, int n) {
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        tw[m] = mk((decltype(tw[0].x))c, (decltype(tw[0].x))s);
    }
}

template <bool INV, class C>
__device__ __forceinline__ C twid(const C* tw, int m) {
    C w = tw[m];
    return INV ? cconj(w) : w;
}

// Out-of-place generic stage (any radix R, read from src, write to dst).
template <bool INV, class C>
__device__ __forceinline__ void stage_generic(const C* src, C* dst, const C* tw, int n, int R,
                                              int Ns, int CB) {
    const int nr = n / R;
    const int step = n / (Ns * R);
    const int nout = n * CB;
    for (int e = threadIdx.x; e < nout; e += blockDim.x) {
        const int c = e % CB, bf = e / CB;
        const int m = bf % R, j = bf / R;  // output m of butterfly j
        const int k = j % Ns;
        C acc = mk((decltype(tw[0].x))0, (decltype(tw[0].x))0);
        // twiddle W_n^{i k step} times DFT factor W_R^{i m} = W_n^{(i m mod R) nr}; both
        // exponents stay below n (k step < n / R, (i m mod R) nr < n), so the sum
        // wraps at most once and the exponents advance by adding, with no division
        const int a_step = k * step;
        int a_tw = 0, im = 0;
        for (int i = 0; i < R; ++i) {
            C x = src[(j + i * nr) * CB + c];
            int q = a_tw + im * nr;
            if (q >= n) q -= n;
            cfma(acc, x, twid<INV>(tw, q));
            a_tw += a_step;
            im += m;
            if (im >= R) im -= R;
        }
        const int base = (j / Ns) * Ns * R + k;
        dst[(base + m * Ns) * CB + c] = acc;
    }
    __syncthreads();
}

// Run a full plan on `buf` with out-of-place generic stages only (ping-pong
// between `buf` and `alt`, both [n][CB]).  Used for line lengths without a
// register codelet; returns the buffer holding the result.
template <bool INV, class C>
__device__ C* fft_tile(C* buf, C* alt, const C* tw, const FftPlan1D& pl, int CB) {
    const int n = pl.n;
    int Ns = 1;
    C* cur = buf;
    C* oth = alt;
    for (int s = 0; s < pl.nstages; ++s) {
        const int R = pl.radix[s];
        stage_generic<INV>(cur, oth, tw, n, R, Ns, CB);
        C* t = cur;
        cur = oth;
        oth = t;
        Ns *= R;
    }
    return cur;
}

}  // namespace cpphf
