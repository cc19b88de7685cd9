// Shared-memory batched 1-D FFT on a tile of n points x CB channels.
//
// The tile is row-major [n][CB] complex in shared memory (channel fastest, so a
// warp touches consecutive 16-byte words).  A plan is a list of radices whose
// product is n; every stage is a Stockham autosort step
//
//   for butterfly j in [0, n/R), channel c:
//       k = j mod Ns;  v_i = x[j + i n/R] * W_n^{i k n/(Ns R)}   (i < R)
//       v = DFT_R(v);  y[(j/Ns) Ns R + k + i Ns] = v_i,           Ns *= R
//
// executed in place: each thread loads all its butterflies' inputs into
// registers, the block synchronises, then writes the outputs.  Radices 2, 3, 4,
// 5, 7 and 8 run from registers; any other prime factor runs as an
// out-of-place direct DFT stage through a second tile buffer.  Twiddles are one
// table W_n^m = exp(-2 pi i m / n), m < n, built per block with sincospi().
#pragma once

#include "common.cuh"

namespace cpphf {

constexpr int kMaxStages = 24;
constexpr int kEptMax = 16;  // tile elements per thread the register stages are sized for

struct FftPlan1D {
    int n;
    int nstages;
    int generic;  // 1 if some stage uses the out-of-place generic radix
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

// In-register DFT of size R (forward sign -1, inverse +1).  `tw` is the n-point
// table, `nr` = n / R gives W_R^q = W_n^{q nr}.
template <int R, bool INV, class C>
__device__ __forceinline__ void dft_reg(C (&v)[R], const C* tw, int nr) {
    constexpr int S = INV ? 1 : -1;
    using Rt = decltype(v[0].x);
    if constexpr (R == 1) {
        return;
    } else if constexpr (R == 2) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const Rt h = (Rt)0.86602540378443864676;  // sqrt(3)/2
        C a = v[0], t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
        C m = mk(a.x - (Rt)0.5 * t1.x, a.y - (Rt)0.5 * t1.y);
        C r = cmuli<S>(cscale(t2, h));
        v[0] = cadd(a, t1);
        v[1] = cadd(m, r);
        v[2] = csub(m, r);
    } else if constexpr (R == 4) {
        C a = v[0], b = v[1], c = v[2], d = v[3];
        C s0 = cadd(a, c), d0 = csub(a, c), s1 = cadd(b, d), d1 = cmuli<S>(csub(b, d));
        v[0] = cadd(s0, s1);
        v[1] = cadd(d0, d1);
        v[2] = csub(s0, s1);
        v[3] = csub(d0, d1);
    } else if constexpr (R == 8) {
        const Rt q = (Rt)0.70710678118654752440;  // sqrt(2)/2
        C e[4] = {v[0], v[2], v[4], v[6]};
        C o[4] = {v[1], v[3], v[5], v[7]};
        dft_reg<4, INV>(e, tw, 0);
        dft_reg<4, INV>(o, tw, 0);
        // W8^m = exp(S 2 pi i m / 8)
        C o1 = mk((o[1].x - (Rt)S * o[1].y) * q, (o[1].y + (Rt)S * o[1].x) * q);
        C o2 = cmuli<S>(o[2]);
        C o3 = mk((-o[3].x - (Rt)S * o[3].y) * q, (-o[3].y + (Rt)S * o[3].x) * q);
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    } else {
        // generic small odd radix from the twiddle table
        C out[R];
#pragma unroll
        for (int m = 0; m < R; ++m) {
            C acc = v[0];
#pragma unroll
            for (int i = 1; i < R; ++i) {
                const int q = (i * m) % R;
                cfma(acc, v[i], twid<INV>(tw, q * nr));
            }
            out[m] = acc;
        }
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = out[m];
    }
}

// One in-place Stockham stage of radix R on the [n][CB] tile.
template <int R, bool INV, class C>
__device__ __forceinline__ void stage_reg(C* buf, const C* tw, int n, int Ns, int CB) {
    constexpr int BMAX = (kEptMax + R - 1) / R;
    const int nr = n / R;
    const int nbf = nr * CB;
    const int step = n / (Ns * R);
    C v[BMAX][R];
#pragma unroll
    for (int b = 0; b < BMAX; ++b) {
        const int bf = threadIdx.x + b * blockDim.x;
        if (bf < nbf) {
            const int c = bf % CB, j = bf / CB;
#pragma unroll
            for (int i = 0; i < R; ++i) v[b][i] = buf[(j + i * nr) * CB + c];
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < BMAX; ++b) {
        const int bf = threadIdx.x + b * blockDim.x;
        if (bf < nbf) {
            const int c = bf % CB, j = bf / CB;
            const int k = j % Ns;
#pragma unroll
            for (int i = 1; i < R; ++i) {
                if (k != 0) v[b][i] = cmul(v[b][i], twid<INV>(tw, i * k * step));
            }
            dft_reg<R, INV>(v[b], tw, nr);
            const int base = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int i = 0; i < R; ++i) buf[(base + i * Ns) * CB + c] = v[b][i];
        }
    }
    __syncthreads();
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
        for (int i = 0; i < R; ++i) {
            C x = src[(j + i * nr) * CB + c];
            // twiddle W_n^{i k step} then DFT factor W_R^{i m} = W_n^{(i m mod R) nr}
            const long long q = ((long long)i * k * step + (long long)((i * m) % R) * nr) % n;
            cfma(acc, x, twid<INV>(tw, (int)q));
        }
        const int base = (j / Ns) * Ns * R + k;
        dst[(base + m * Ns) * CB + c] = acc;
    }
    __syncthreads();
}

// Run a full plan on `buf`.  `alt` (may be null when !pl.generic) is the
// second tile buffer.  Returns the buffer that holds the result.
template <bool INV, class C>
__device__ C* fft_tile(C* buf, C* alt, const C* tw, const FftPlan1D& pl, int CB) {
    const int n = pl.n;
    int Ns = 1;
    C* cur = buf;
    C* oth = alt;
    for (int s = 0; s < pl.nstages; ++s) {
        const int R = pl.radix[s];
        switch (R) {
            case 2: stage_reg<2, INV>(cur, tw, n, Ns, CB); break;
            case 3: stage_reg<3, INV>(cur, tw, n, Ns, CB); break;
            case 4: stage_reg<4, INV>(cur, tw, n, Ns, CB); break;
            case 5: stage_reg<5, INV>(cur, tw, n, Ns, CB); break;
            case 7: stage_reg<7, INV>(cur, tw, n, Ns, CB); break;
            case 8: stage_reg<8, INV>(cur, tw, n, Ns, CB); break;
            default: {
                stage_generic<INV>(cur, oth, tw, n, R, Ns, CB);
                C* t = cur;
                cur = oth;
                oth = t;
            }
        }
        Ns *= R;
    }
    return cur;
}

}  // namespace cpphf
