// Exchange self-energy  Sigma(k) = -IFFT2[ FFT2(P - refP) . VR ]  on a (nk1, nk2)
// mesh with nb*nb channel-interleaved orbital pairs (cpp_hf selfenergy.hpp:60-171).
//
// Three passes over an (nk1, nk2, C) intermediate T, each a grid of CTAs that
// owns one full FFT line for a block of CB consecutive channels:
//   A  rows:    load P[kx, :, chunk] (- refP), FFT along ky              -> T
//   B  columns: load T[:, ky, chunk], FFT along kx, * VR, IFFT along kx   -> T
//               (optional ifftshift of the kx axis applied on the store)
//   C  rows:    load T[kx, :, chunk], IFFT along ky, * (-1/(nk1 nk2))     -> Sigma
//               (optional ifftshift of ky; HCP unpack + conjugate mirror)
// For the full FP64 path T aliases Sigma (every CTA reads its whole tile
// before writing it), so the compulsory DRAM traffic is P + VR + Sigma and the
// intermediate round trips go through L2 (P and VR are streamed with
// evict-first loads).  HCP (upper-triangle packing) and the complex64 form use
// a workspace field for T.
//
// Line lengths with a register codelet (fft_reg.cuh: 1..6, 8, 9, 12, 16, 18,
// 24, 32, 36, 48, 64, 72, 96, 128, 144, 192, 256, 288) run the four-step
// transform with global loads/stores straight from/to registers and one
// shared-memory transpose per direction; any other length runs the generic
// out-of-place Stockham stages of fft.cuh.
#include "common.cuh"
#include "exchange.cuh"
#include "fft.cuh"
#include "fft_reg.cuh"
#include "bulk.cuh"
#include "exchange_pipe.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>

namespace cpphf {

namespace {

constexpr int kTargetThreads = 256;

// column-pass modes: multiply by VR (the exchange), by conj(VR) (its adjoint),
// or stop after the forward transform (2-D FFT of the input, for dL/dVR)
constexpr int kColsVR = 0;
constexpr int kColsConjVR = 1;
constexpr int kColsForwardOnly = 2;

// channel -> (row, col) of the HCP packing (upper triangle, row-major).
__device__ __forceinline__ void hcp_pair(int ch, int nb, int& i, int& j) {
    int r = 0, c = ch;
    while (c >= nb - r) {
        c -= nb - r;
        ++r;
    }
    i = r;
    j = r + c;
}

__device__ __forceinline__ void build_map(int* map, int chunk0, int CB, int C, int nb, int hcp) {
    for (int c = threadIdx.x; c < CB; c += blockDim.x) {
        const int ch = chunk0 + c;
        int off = -1, mir = -1;
        if (ch < C) {
            if (hcp) {
                int i, j;
                hcp_pair(ch, nb, i, j);
                off = i * nb + j;
                mir = (i != j) ? j * nb + i : -1;
            } else {
                off = ch;
            }
        }
        map[2 * c] = off;
        map[2 * c + 1] = mir;
    }
}

template <class Cx>
__device__ __forceinline__ Cx czero() {
    return mk((decltype(Cx{}.x))0, (decltype(Cx{}.x))0);
}

// ===========================================================================
// Specialised four-step kernels (N = N1 * N2 with register codelets)
// smem: tw[N] | S[N * CB] | map[2 * CB]
// ===========================================================================
template <class Cx>
struct SView {
    Cx* tw;
    Cx* S;
    int* map;
    __device__ SView(unsigned char* base, int N, int CB) {
        tw = reinterpret_cast<Cx*>(base);
        S = tw + N;
        map = reinterpret_cast<int*>(S + (size_t)N * CB);
    }
};

template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(256) k_rows_fwd_s(const double2* __restrict__ P, const double2* __restrict__ refP,
                                                     Cx* T, ExchangeGeom g, int CB) {
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SView<Cx> s(smem_raw, N, CB);
    const int kx = blockIdx.x, chunk0 = blockIdx.y * CB;
    const int c = threadIdx.x % CB, a = threadIdx.x / CB;
    build_line_twiddles(s.tw, N);
    build_map(s.map, chunk0, CB, g.C, g.nb, g.hcp);
    __syncthreads();
    const size_t nb2 = (size_t)g.nb * g.nb;
    const int off = s.map[2 * c];
    if (a < N2) {
        Cx v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
            double2 x = mk(0.0, 0.0);
            if (off >= 0) {
                const size_t idx = ((size_t)kx * g.n1 + (N2 * n1 + a)) * nb2 + off;
                x = ld_stream(P + idx);
                if (refP) x = csub(x, ld_stream(refP + idx));
            }
            v[n1] = to_c(x, Cx{});
        }
        dft<N1, false>(v);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) s.S[(k1 * N2 + a) * CB + c] = cmul(v[k1], s.tw[a * k1]);
    }
    __syncthreads();
    if (a < N1) {
        Cx u[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) u[n2] = s.S[(a * N2 + n2) * CB + c];
        dft<N2, false>(u);
        const int ch = chunk0 + c;
        if (ch < g.C) {
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) st_l2(T + ((size_t)kx * g.n1 + (a + N1 * k2)) * g.Ct + ch, u[k2]);
        }
    }
}

template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(256) k_cols_conv_s(Cx* T, const double2* __restrict__ VR, ExchangeGeom g, int CB,
                                                      int vmode) {
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SView<Cx> s(smem_raw, N, CB);
    const int ky = blockIdx.x, chunk0 = blockIdx.y * CB;
    const int c = threadIdx.x % CB, a = threadIdx.x / CB;
    const int ch = chunk0 + c;
    const bool live = ch < g.C;
    build_line_twiddles(s.tw, N);
    __syncthreads();
    if (a < N2) {
        Cx v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1)
            v[n1] = live ? ld_l2(T + ((size_t)(N2 * n1 + a) * g.n1 + ky) * g.Ct + ch) : czero<Cx>();
        dft<N1, false>(v);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) s.S[(k1 * N2 + a) * CB + c] = cmul(v[k1], s.tw[a * k1]);
    }
    __syncthreads();
    Cx u[N2];
    if (a < N1) {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) u[n2] = s.S[(a * N2 + n2) * CB + c];
        dft<N2, false>(u);
        if (vmode == kColsForwardOnly) {
            // u[k2] = X[a + N1 k2]: the 2-D forward transform, stored in natural order
            if (live) {
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) st_l2(T + ((size_t)(a + N1 * k2) * g.n1 + ky) * g.Ct + ch, u[k2]);
            }
        } else {
            // u[k2] = X[a + N1 k2]: multiply by VR (or conj VR) at kx = a + N1 k2
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) {
                if (live) {
                    const size_t vi = ((size_t)(a + N1 * k2) * g.n1 + ky) * g.dv + (g.dv == 1 ? 0 : ch);
                    double2 w = ld_stream(VR + vi);
                    if (vmode == kColsConjVR) w = cconj(w);
                    u[k2] = cmul(u[k2], to_c(w, Cx{}));
                }
            }
            dft<N2, true>(u);
        }
    }
    if (vmode == kColsForwardOnly) return;
    __syncthreads();
    if (a < N1) {
#pragma unroll
        for (int na = 0; na < N2; ++na) s.S[(a * N2 + na) * CB + c] = cmulc(u[na], s.tw[na * a]);
    }
    __syncthreads();
    if (a < N2) {
        Cx v[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) v[k1] = s.S[(k1 * N2 + a) * CB + c];
        dft<N1, true>(v);
        if (live) {
            const int s0 = g.shift ? g.n0 / 2 : 0;
#pragma unroll
            for (int nbx = 0; nbx < N1; ++nbx) {
                const int kx = a + N2 * nbx;
                const int dx = (kx - s0 + g.n0) % g.n0;
                st_l2(T + ((size_t)dx * g.n1 + ky) * g.Ct + ch, v[nbx]);
            }
        }
    }
}

template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(256) k_rows_inv_s(const Cx* T, double2* Sigma, ExchangeGeom g, int CB, double scale) {
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SView<Cx> s(smem_raw, N, CB);
    const int kx = blockIdx.x, chunk0 = blockIdx.y * CB;
    const int c = threadIdx.x % CB, a = threadIdx.x / CB;
    const int ch = chunk0 + c;
    const bool live = ch < g.C;
    build_line_twiddles(s.tw, N);
    build_map(s.map, chunk0, CB, g.C, g.nb, g.hcp);
    __syncthreads();
    if (a < N1) {
        Cx u[N2];
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2)
            u[k2] = live ? ld_l2(T + ((size_t)kx * g.n1 + (a + N1 * k2)) * g.Ct + ch) : czero<Cx>();
        dft<N2, true>(u);
#pragma unroll
        for (int na = 0; na < N2; ++na) s.S[(a * N2 + na) * CB + c] = cmulc(u[na], s.tw[na * a]);
    }
    __syncthreads();
    if (a < N2) {
        Cx v[N1];
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) v[k1] = s.S[(k1 * N2 + a) * CB + c];
        dft<N1, true>(v);
        const int off = s.map[2 * c], mir = s.map[2 * c + 1];
        if (off >= 0) {
            const size_t nb2 = (size_t)g.nb * g.nb;
            const int s1 = g.shift ? g.n1 / 2 : 0;
#pragma unroll
            for (int nbx = 0; nbx < N1; ++nbx) {
                const int ky = a + N2 * nbx;
                const int dy = (ky - s1 + g.n1) % g.n1;
                const double2 val = cscale(to_d(v[nbx]), scale);
                double2* dst = Sigma + ((size_t)kx * g.n1 + dy) * nb2;
                dst[off] = val;
                if (mir >= 0) dst[mir] = cconj(val);
            }
        }
    }
}


// ===========================================================================
// Pipelined four-step kernels (full channel set, no HCP).  Persistent CTAs
// walk the tiles (line, channel chunk) with a stride of gridDim.x; thread 0
// keeps the next nst-1 tiles in flight (TMA tensor copies into a ring of nst
// shared-memory stages) while the CTA transforms the current one.  The
// transpose of the four-step runs in place in the current stage.
// smem: tw[N] | mbar[kMaxPipeStages] | stage[nst] = { in tile [N][CB] (double2,
//       or Cx for T), second tile [N][CB] double2 (refP or VR) }
// ===========================================================================
// Columns pass: the T tiles keep the ring of nst stages, VR has one buffer that
// is refilled for the next tile as soon as the current tile's multiply has read
// it (VR is read once per tile, in the middle of the transform).
// The twiddle table holds w^m for m < N/2 when N is even (w^(m + N/2) = -w^m),
// which keeps a 192-point line at three CTAs per SM.
// smem: tw[N/2 or N] | mbar[kMaxPipeStages + 1] | T stage[nst] | VR [N][CB] double2
struct ColsLayout {
    size_t tw, bar, stage0, stage_bytes, vr, total;
};

__host__ __device__ constexpr int cols_twiddles(int N) { return (N % 2 == 0) ? N / 2 : N; }

__host__ __device__ inline ColsLayout cols_layout(int N, int CB, size_t in_elem, int nst) {
    ColsLayout L;
    L.tw = 0;
    L.bar = (sizeof(double2) * (size_t)cols_twiddles(N) + 15) & ~(size_t)15;
    L.stage0 = (L.bar + 8 * (kMaxPipeStages + 1) + 127) & ~(size_t)127;
    L.stage_bytes = ((in_elem * (size_t)N * CB) + 127) & ~(size_t)127;
    L.vr = L.stage0 + (size_t)nst * L.stage_bytes;
    L.total = L.vr + ((sizeof(double2) * (size_t)N * CB + 127) & ~(size_t)127) + 128;
    return L;
}

// pass A: rows forward.  Tile t -> (kx = t / nchunk, chunk = t % nchunk).
template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(256, 2) k_rows_fwd_p(const __grid_constant__ CUtensorMap mP,
                                                       const __grid_constant__ CUtensorMap mR, int has_refP, Cx* T,
                                                       ExchangeGeom g, int CB, int nchunk, int ntiles, int nst) {
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char* smem_raw = align128(smem_dyn);
    const bool has_ref = has_refP != 0;
    const PipeLayout L = pipe_layout(N, CB, sizeof(double2), has_ref, nst);
    Cx* tw = reinterpret_cast<Cx*>(smem_raw + L.tw);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw + L.bar);
    const int c = threadIdx.x % CB, a = threadIdx.x / CB;
    build_line_twiddles(tw, N);
    if (threadIdx.x == 0) {
        for (int b = 0; b < nst; ++b) mbar_init(&bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int stage) {
        if (threadIdx.x != 0) return;
        const int kx = t / nchunk, c0 = (t - kx * nchunk) * CB;
        const unsigned box = (unsigned)(N * CB * sizeof(double2));
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[stage], box * (has_ref ? 2u : 1u));
        tma_load_3d(st, &mP, 2 * c0, 0, kx, &bar[stage]);
        if (has_ref) tma_load_3d(st + L.in_bytes, &mR, 2 * c0, 0, kx, &bar[stage]);
    };
    int i = 0;
    for (int j = 0; j < nst - 1; ++j)
        if ((int)blockIdx.x + j * (int)gridDim.x < ntiles) issue(blockIdx.x + j * gridDim.x, j);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
        const int stage = i % nst;
        {
            const int ahead = t + (nst - 1) * (int)gridDim.x;
            if (ahead < ntiles) issue(ahead, (i + nst - 1) % nst);
        }
        if (!mbar_wait(&bar[stage], (unsigned)((i / nst) & 1), g.err)) return;
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        const double2* in = reinterpret_cast<const double2*>(st);
        const double2* rin = reinterpret_cast<const double2*>(st + L.in_bytes);
        const int kx = t / nchunk, c0 = (t - kx * nchunk) * CB;
        Cx v[N1];
        if (a < N2) {
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) {
                double2 x = in[(N2 * n1 + a) * CB + c];
                if (has_ref) x = csub(x, rin[(N2 * n1 + a) * CB + c]);
                v[n1] = to_c(x, Cx{});
            }
            dft<N1, false>(v);
        }
        __syncthreads();
        Cx* S = reinterpret_cast<Cx*>(st);
        if (a < N2) {
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) S[(k1 * N2 + a) * CB + c] = cmul(v[k1], tw[a * k1]);
        }
        __syncthreads();
        if (a < N1) {
            Cx u[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) u[n2] = S[(a * N2 + n2) * CB + c];
            dft<N2, false>(u);
            const int ch = c0 + c;
            if (ch < g.C) {
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) st_l2(T + ((size_t)kx * g.n1 + (a + N1 * k2)) * g.Ct + ch, u[k2]);
            }
        }
        __syncthreads();
    }
}

// pass B: columns forward, * VR, inverse.  Tile t -> (ky, chunk).  At most 128
// threads per CTA; three CTAs per SM for lines of up to 192 points.
template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(kColsMaxThreads, (N1 * N2 <= 192 ? 3 : 1))
    k_cols_conv_p(const __grid_constant__ CUtensorMap mT, const __grid_constant__ CUtensorMap mV, Cx* T,
                  ExchangeGeom g, int CB, int nchunk, int ntiles, int conjv, int nst) {
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char* smem_raw = align128(smem_dyn);
    const ColsLayout L = cols_layout(N, CB, sizeof(Cx), nst);
    Cx* tw = reinterpret_cast<Cx*>(smem_raw + L.tw);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw + L.bar);
    unsigned long long* barV = bar + kMaxPipeStages;
    const double2* Vt = reinterpret_cast<const double2*>(smem_raw + L.vr);
    const int c = threadIdx.x % CB, a = threadIdx.x / CB;
    constexpr int NTW = cols_twiddles(N);
    using R = decltype(Cx{}.x);
    for (int m = threadIdx.x; m < NTW; m += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * (double)m / (double)N, &sn, &cs);
        tw[m] = mk((R)cs, (R)sn);
    }
    auto twv = [&](int j) -> Cx {
        if (NTW == N || j < NTW) return tw[j];
        const Cx v = tw[j - NTW];
        return mk(-v.x, -v.y);
    };
    if (threadIdx.x == 0) {
        for (int b = 0; b < nst; ++b) mbar_init(&bar[b], 1);
        mbar_init(barV, 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int stage) {
        if (threadIdx.x != 0) return;
        const int ky = t / nchunk, c0 = (t - ky * nchunk) * CB;
        const unsigned boxT = (unsigned)(N * CB * sizeof(Cx));
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[stage], boxT);
        tma_load_3d(st, &mT, 2 * c0, ky, 0, &bar[stage]);
    };
    auto issue_vr = [&](int t) {
        if (threadIdx.x != 0) return;
        const int ky = t / nchunk, c0 = (t - ky * nchunk) * CB;
        const unsigned boxV = (unsigned)(N * (g.dv == 1 ? 1 : CB) * sizeof(double2));
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(barV, boxV);
        tma_load_3d(smem_raw + L.vr, &mV, g.dv == 1 ? 0 : 2 * c0, ky, 0, barV);
    };
    const int s0 = g.shift ? g.n0 / 2 : 0;
    int i = 0;
    for (int j = 0; j < nst - 1; ++j)
        if ((int)blockIdx.x + j * (int)gridDim.x < ntiles) issue(blockIdx.x + j * gridDim.x, j);
    if ((int)blockIdx.x < ntiles) issue_vr(blockIdx.x);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
        const int stage = i % nst;
        {
            const int ahead = t + (nst - 1) * (int)gridDim.x;
            if (ahead < ntiles) issue(ahead, (i + nst - 1) % nst);
        }
        if (!mbar_wait(&bar[stage], (unsigned)((i / nst) & 1), g.err)) return;
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        Cx* S = reinterpret_cast<Cx*>(st);
        const int ky = t / nchunk, c0 = (t - ky * nchunk) * CB;
        const int ch = c0 + c;
        Cx v[N1];
        if (a < N2) {
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) v[n1] = S[(N2 * n1 + a) * CB + c];
            dft<N1, false>(v);
        }
        __syncthreads();
        if (a < N2) {
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) S[(k1 * N2 + a) * CB + c] = cmul(v[k1], twv(a * k1));
        }
        __syncthreads();
        Cx u[N2];
        if (a < N1) {
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) u[n2] = S[(a * N2 + n2) * CB + c];
            dft<N2, false>(u);
        }
        if (!mbar_wait(barV, (unsigned)(i & 1), g.err)) return;  // this tile's VR
        if (a < N1) {
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) {
                double2 w = g.dv == 1 ? Vt[a + N1 * k2] : Vt[(a + N1 * k2) * CB + c];
                if (conjv) w = cconj(w);
                u[k2] = cmul(u[k2], to_c(w, Cx{}));
            }
            dft<N2, true>(u);
        }
        __syncthreads();
        if (t + (int)gridDim.x < ntiles) issue_vr(t + gridDim.x);  // every read of VR is done
        if (a < N1) {
#pragma unroll
            for (int na = 0; na < N2; ++na) S[(a * N2 + na) * CB + c] = cmulc(u[na], twv(na * a));
        }
        __syncthreads();
        if (a < N2) {
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) v[k1] = S[(k1 * N2 + a) * CB + c];
            dft<N1, true>(v);
            if (ch < g.C) {
#pragma unroll
                for (int nbx = 0; nbx < N1; ++nbx) {
                    const int kx = a + N2 * nbx;
                    const int dx = (kx - s0 + g.n0) % g.n0;
                    st_l2(T + ((size_t)dx * g.n1 + ky) * g.Ct + ch, v[nbx]);
                }
            }
        }
        __syncthreads();
    }
}

// pass C: rows inverse, scale, shift, store Sigma.  Tile t -> (kx, chunk).
template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(256, 2) k_rows_inv_p(const __grid_constant__ CUtensorMap mT, double2* Sigma,
                                                       ExchangeGeom g, int CB, int nchunk, int ntiles, double scale,
                                                       int nst) {
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char* smem_raw = align128(smem_dyn);
    const PipeLayout L = pipe_layout(N, CB, sizeof(Cx), false, nst);
    Cx* tw = reinterpret_cast<Cx*>(smem_raw + L.tw);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw + L.bar);
    const int c = threadIdx.x % CB, a = threadIdx.x / CB;
    const size_t nb2 = (size_t)g.nb * g.nb;
    build_line_twiddles(tw, N);
    if (threadIdx.x == 0) {
        for (int b = 0; b < nst; ++b) mbar_init(&bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int stage) {
        if (threadIdx.x != 0) return;
        const int kx = t / nchunk, c0 = (t - kx * nchunk) * CB;
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[stage], (unsigned)(N * CB * sizeof(Cx)));
        tma_load_3d(st, &mT, 2 * c0, 0, kx, &bar[stage]);
    };
    const int s1 = g.shift ? g.n1 / 2 : 0;
    int i = 0;
    for (int j = 0; j < nst - 1; ++j)
        if ((int)blockIdx.x + j * (int)gridDim.x < ntiles) issue(blockIdx.x + j * gridDim.x, j);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
        const int stage = i % nst;
        {
            const int ahead = t + (nst - 1) * (int)gridDim.x;
            if (ahead < ntiles) issue(ahead, (i + nst - 1) % nst);
        }
        if (!mbar_wait(&bar[stage], (unsigned)((i / nst) & 1), g.err)) return;
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        Cx* S = reinterpret_cast<Cx*>(st);
        const int kx = t / nchunk, c0 = (t - kx * nchunk) * CB;
        const int ch = c0 + c;
        Cx u[N2];
        if (a < N1) {
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) u[k2] = S[(a + N1 * k2) * CB + c];
            dft<N2, true>(u);
        }
        __syncthreads();
        if (a < N1) {
#pragma unroll
            for (int na = 0; na < N2; ++na) S[(a * N2 + na) * CB + c] = cmulc(u[na], tw[na * a]);
        }
        __syncthreads();
        if (a < N2) {
            Cx v[N1];
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) v[k1] = S[(k1 * N2 + a) * CB + c];
            dft<N1, true>(v);
            if (ch < g.C) {
#pragma unroll
                for (int nbx = 0; nbx < N1; ++nbx) {
                    const int ky = a + N2 * nbx;
                    const int dy = (ky - s1 + g.n1) % g.n1;
                    Sigma[((size_t)kx * g.n1 + dy) * nb2 + ch] = cscale(to_d(v[nbx]), scale);
                }
            }
        }
        __syncthreads();
    }
}

// ===========================================================================
// Generic kernels (any line length)
// smem: tw[n] | buf[n * CB] | alt[n * CB] | map[2 * CB]
// ===========================================================================
template <class Cx>
struct GView {
    Cx* tw;
    Cx* buf;
    Cx* alt;
    int* map;
    __device__ GView(unsigned char* base, int n, int CB) {
        tw = reinterpret_cast<Cx*>(base);
        buf = tw + n;
        alt = buf + (size_t)n * CB;
        map = reinterpret_cast<int*>(alt + (size_t)n * CB);
    }
};

template <class Cx>
__global__ void k_rows_fwd_g(const double2* __restrict__ P, const double2* __restrict__ refP, Cx* T, ExchangeGeom g,
                             FftPlan1D pl, int CB) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GView<Cx> s(smem_raw, pl.n, CB);
    const int kx = blockIdx.x, chunk0 = blockIdx.y * CB, n = pl.n;
    build_twiddles(s.tw, n);
    build_map(s.map, chunk0, CB, g.C, g.nb, g.hcp);
    __syncthreads();
    const size_t nb2 = (size_t)g.nb * g.nb;
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int ny = e / CB, c = e - ny * CB;
        const int off = s.map[2 * c];
        double2 v = mk(0.0, 0.0);
        if (off >= 0) {
            const size_t idx = ((size_t)kx * g.n1 + ny) * nb2 + off;
            v = ld_stream(P + idx);
            if (refP) v = csub(v, ld_stream(refP + idx));
        }
        s.buf[e] = to_c(v, Cx{});
    }
    __syncthreads();
    Cx* r = fft_tile<false>(s.buf, s.alt, s.tw, pl, CB);
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int ny = e / CB, c = e - ny * CB;
        const int ch = chunk0 + c;
        if (ch < g.C) st_l2(T + ((size_t)kx * g.n1 + ny) * g.Ct + ch, r[e]);
    }
}

template <class Cx>
__global__ void k_cols_conv_g(Cx* T, const double2* __restrict__ VR, ExchangeGeom g, FftPlan1D pl, int CB,
                              int vmode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GView<Cx> s(smem_raw, pl.n, CB);
    const int ky = blockIdx.x, chunk0 = blockIdx.y * CB, n = pl.n;
    build_twiddles(s.tw, n);
    __syncthreads();
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int nx = e / CB, c = e - nx * CB;
        const int ch = chunk0 + c;
        s.buf[e] = (ch < g.C) ? ld_l2(T + ((size_t)nx * g.n1 + ky) * g.Ct + ch) : czero<Cx>();
    }
    __syncthreads();
    Cx* r = fft_tile<false>(s.buf, s.alt, s.tw, pl, CB);
    if (vmode == kColsForwardOnly) {
        for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
            const int nx = e / CB, c = e - nx * CB;
            const int ch = chunk0 + c;
            if (ch < g.C) st_l2(T + ((size_t)nx * g.n1 + ky) * g.Ct + ch, r[e]);
        }
        return;
    }
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int nx = e / CB, c = e - nx * CB;
        const int ch = chunk0 + c;
        if (ch < g.C) {
            const size_t vi = ((size_t)nx * g.n1 + ky) * g.dv + (g.dv == 1 ? 0 : ch);
            double2 w = ld_stream(VR + vi);
            if (vmode == kColsConjVR) w = cconj(w);
            r[e] = cmul(r[e], to_c(w, Cx{}));
        }
    }
    __syncthreads();
    Cx* q = fft_tile<true>(r, r == s.buf ? s.alt : s.buf, s.tw, pl, CB);
    const int s0 = g.shift ? g.n0 / 2 : 0;
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int nx = e / CB, c = e - nx * CB;
        const int ch = chunk0 + c;
        const int dx = (nx - s0 + g.n0) % g.n0;
        if (ch < g.C) st_l2(T + ((size_t)dx * g.n1 + ky) * g.Ct + ch, q[e]);
    }
}

template <class Cx>
__global__ void k_rows_inv_g(const Cx* T, double2* Sigma, ExchangeGeom g, FftPlan1D pl, int CB, double scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GView<Cx> s(smem_raw, pl.n, CB);
    const int kx = blockIdx.x, chunk0 = blockIdx.y * CB, n = pl.n;
    build_twiddles(s.tw, n);
    build_map(s.map, chunk0, CB, g.C, g.nb, g.hcp);
    __syncthreads();
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int ny = e / CB, c = e - ny * CB;
        const int ch = chunk0 + c;
        s.buf[e] = (ch < g.C) ? ld_l2(T + ((size_t)kx * g.n1 + ny) * g.Ct + ch) : czero<Cx>();
    }
    __syncthreads();
    Cx* r = fft_tile<true>(s.buf, s.alt, s.tw, pl, CB);
    const size_t nb2 = (size_t)g.nb * g.nb;
    const int s1 = g.shift ? g.n1 / 2 : 0;
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int ny = e / CB, c = e - ny * CB;
        const int off = s.map[2 * c];
        if (off < 0) continue;
        const int dy = (ny - s1 + g.n1) % g.n1;
        const double2 v = cscale(to_d(r[e]), scale);
        double2* dst = Sigma + ((size_t)kx * g.n1 + dy) * nb2;
        dst[off] = v;
        const int mir = s.map[2 * c + 1];
        if (mir >= 0) dst[mir] = cconj(v);
    }
}

// ===========================================================================
// launch plumbing
// ===========================================================================
struct Launch {
    int CB;
    int threads;
    size_t smem;
    int nchunk;
};

// channels per tile so that a CTA has about `target` threads; chunks balanced.
Launch plan_launch(int lanes, int C, size_t elem, int n, bool generic, int target = kTargetThreads) {
    Launch L;
    const int cbmax = std::max(1, std::min(C, target / std::max(lanes, 1)));
    const int nch = (C + cbmax - 1) / cbmax;
    L.CB = (C + nch - 1) / nch;
    L.nchunk = (C + L.CB - 1) / L.CB;
    int threads = generic ? std::min(1024, std::max(64, n * L.CB)) : lanes * L.CB;
    threads = std::min(1024, ((threads + 31) / 32) * 32);
    L.threads = threads;
    L.smem = elem * (size_t)n + elem * (size_t)n * L.CB * (generic ? 2 : 1) + sizeof(int) * 2 * (size_t)L.CB;
    return L;
}


// Pipelined-pass shape: threads per CTA (sets the channels per tile) and the
// number of shared-memory stages.  Block shapes of 64-256 threads and 2-4
// stages were swept on the 192x192, nb = 8 workload; 128 x 2 is the fastest
// for both pass kinds.
struct PipeCfg {
    int threads;
    int nst;
};

constexpr PipeCfg kRowsCfg{128, 2};
constexpr PipeCfg kColsCfg{128, 2};

template <class Cx, int N1, int N2>
struct Spec {
    static void attrs() {
        static std::once_flag once;
        std::call_once(once, [] {
            raise_smem(k_rows_fwd_s<Cx, N1, N2>);
            raise_smem(k_cols_conv_s<Cx, N1, N2>);
            raise_smem(k_rows_inv_s<Cx, N1, N2>);
            raise_smem(k_rows_fwd_p<Cx, N1, N2>);
            raise_smem(k_cols_conv_p<Cx, N1, N2>);
            raise_smem(k_rows_inv_p<Cx, N1, N2>);
        });
    }
    // persistent grid size for a pipelined kernel with `smem` bytes
    template <class K>
    static int pgrid(K kern, int threads, size_t smem, int ntiles) {
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem);
        (void)cudaGetLastError();
        if (per < 1) per = 1;
        return std::max(1, std::min(ntiles, per * num_sms()));
    }
    // TMA boxes need 16-byte multiples for the inner extent, the row stride and
    // the x coordinate (2 c0 scalars): for complex64 T that means even CB and Ct.
    static Launch pipe_launch(const ExchangeGeom& g, const PipeCfg& cfg) {
        return plan_launch(N1 > N2 ? N1 : N2, g.C, sizeof(Cx), N1 * N2, false, cfg.threads);
    }
    static bool pipelined(const ExchangeGeom& g, const PipeCfg& cfg) {
        if (g.hcp || N1 * N2 > 256) return false;
        const Launch L = pipe_launch(g, cfg);
        if (L.threads > 256) return false;  // __launch_bounds__(256)
        if (sizeof(Cx) == 8 && ((L.CB % 2) != 0 || (g.Ct % 2) != 0)) return false;
        return true;
    }
    static CUtensorMapDataType tdt() { return sizeof(Cx) == 16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
    // field (n0, n1, C complex) as a 3-D tensor {2C scalars, n1, n0}
    static bool field_map(CUtensorMap* m, const void* base, CUtensorMapDataType dt, size_t scal, int C,
                          const ExchangeGeom& g, unsigned b0, unsigned b1, unsigned b2) {
        const unsigned long long row = 2ull * C * scal;
        return make_tensor_map_3d(m, base, dt, 2ull * C, (unsigned long long)g.n1, (unsigned long long)g.n0, row,
                                  row * (unsigned long long)g.n1, b0, b1, b2);
    }
    static int rows_fwd(const double2* P, const double2* refP, Cx* T, const ExchangeGeom& g, cudaStream_t st) {
        attrs();
        const PipeCfg cfg = kRowsCfg;
        if (pipelined(g, cfg)) {
            const Launch L = pipe_launch(g, cfg);
            const PipeLayout PL = pipe_layout(N1 * N2, L.CB, sizeof(double2), refP != nullptr, cfg.nst);
            if (PL.total <= kSmemMax) {
                CUtensorMap mP, mR;
                const int nb2 = g.nb * g.nb;
                bool ok = field_map(&mP, P, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, nb2, g, 2 * L.CB, N1 * N2, 1);
                ok = ok && field_map(&mR, refP ? refP : P, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, nb2, g, 2 * L.CB,
                                     N1 * N2, 1);
                if (ok) {
                    const int nt = g.n0 * L.nchunk;
                    const int grid = pgrid(k_rows_fwd_p<Cx, N1, N2>, L.threads, PL.total, nt);
                    k_rows_fwd_p<Cx, N1, N2><<<grid, L.threads, PL.total, st>>>(mP, mR, refP != nullptr, T, g, L.CB,
                                                                                L.nchunk, nt, cfg.nst);
                    CPPHF_LAUNCH_CHECK("exchange rows forward (pipelined)");
                    return CPPHF_OK;
                }
            }
        }
        const Launch L = plan_launch(N1 > N2 ? N1 : N2, g.C, sizeof(Cx), N1 * N2, false);
        k_rows_fwd_s<Cx, N1, N2><<<dim3(g.n0, L.nchunk), L.threads, L.smem, st>>>(P, refP, T, g, L.CB);
        CPPHF_LAUNCH_CHECK("exchange rows forward");
        return CPPHF_OK;
    }
    static int cols(Cx* T, const double2* VR, const ExchangeGeom& g, int vmode, cudaStream_t st) {
        attrs();
        const PipeCfg cfg = kColsCfg;
        if (pipelined(g, cfg) && vmode != kColsForwardOnly && pipe_launch(g, cfg).threads <= kColsMaxThreads) {
            const Launch L = pipe_launch(g, cfg);
            const ColsLayout PL = cols_layout(N1 * N2, L.CB, sizeof(Cx), cfg.nst);
            if (PL.total <= kSmemMax) {
                CUtensorMap mT, mV;
                bool ok = field_map(&mT, T, tdt(), sizeof(Cx) / 2, g.Ct, g, 2 * L.CB, 1, N1 * N2);
                if (g.dv == 1)
                    ok = ok && field_map(&mV, VR, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, 1, g, 2, 1, N1 * N2);
                else
                    ok = ok && field_map(&mV, VR, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, g.dv, g, 2 * L.CB, 1, N1 * N2);
                if (ok) {
                    const int nt = g.n1 * L.nchunk;
                    const int grid = pgrid(k_cols_conv_p<Cx, N1, N2>, L.threads, PL.total, nt);
                    k_cols_conv_p<Cx, N1, N2><<<grid, L.threads, PL.total, st>>>(mT, mV, T, g, L.CB, L.nchunk, nt,
                                                                                 vmode == kColsConjVR ? 1 : 0,
                                                                                 cfg.nst);
                    CPPHF_LAUNCH_CHECK("exchange columns convolve (pipelined)");
                    return CPPHF_OK;
                }
            }
        }
        const Launch L = plan_launch(N1 > N2 ? N1 : N2, g.C, sizeof(Cx), N1 * N2, false);
        k_cols_conv_s<Cx, N1, N2><<<dim3(g.n1, L.nchunk), L.threads, L.smem, st>>>(T, VR, g, L.CB, vmode);
        CPPHF_LAUNCH_CHECK("exchange columns convolve");
        return CPPHF_OK;
    }
    static int rows_inv(const Cx* T, double2* Sigma, const ExchangeGeom& g, double scale, cudaStream_t st) {
        attrs();
        const PipeCfg cfg = kRowsCfg;
        if (pipelined(g, cfg)) {
            const Launch L = pipe_launch(g, cfg);
            const PipeLayout PL = pipe_layout(N1 * N2, L.CB, sizeof(Cx), false, cfg.nst);
            if (PL.total <= kSmemMax) {
                CUtensorMap mT;
                if (field_map(&mT, T, tdt(), sizeof(Cx) / 2, g.Ct, g, 2 * L.CB, N1 * N2, 1)) {
                    const int nt = g.n0 * L.nchunk;
                    const int grid = pgrid(k_rows_inv_p<Cx, N1, N2>, L.threads, PL.total, nt);
                    k_rows_inv_p<Cx, N1, N2><<<grid, L.threads, PL.total, st>>>(mT, Sigma, g, L.CB, L.nchunk, nt,
                                                                                scale, cfg.nst);
                    CPPHF_LAUNCH_CHECK("exchange rows inverse (pipelined)");
                    return CPPHF_OK;
                }
            }
        }
        const Launch L = plan_launch(N1 > N2 ? N1 : N2, g.C, sizeof(Cx), N1 * N2, false);
        k_rows_inv_s<Cx, N1, N2><<<dim3(g.n0, L.nchunk), L.threads, L.smem, st>>>(T, Sigma, g, L.CB, scale);
        CPPHF_LAUNCH_CHECK("exchange rows inverse");
        return CPPHF_OK;
    }
};

template <class Cx>
struct Gen {
    static void attrs() {
        static std::once_flag once;
        std::call_once(once, [] {
            raise_smem(k_rows_fwd_g<Cx>);
            raise_smem(k_cols_conv_g<Cx>);
            raise_smem(k_rows_inv_g<Cx>);
        });
    }
};

// The generic kernels loop over their tile with a block stride, so any block
// size works: cap it at what the kernel's register use allows.
template <class K>
int cap_threads(K kern, int threads) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) {
        (void)cudaGetLastError();
        return std::min(threads, 256);
    }
    const int m = (fa.maxThreadsPerBlock / 32) * 32;
    return std::max(32, std::min(threads, m));
}




template <class Cx>
int pass_rows_fwd(const double2* P, const double2* refP, Cx* T, const ExchangeGeom& g, cudaStream_t st) {
    switch (g.n1) {
#define X(N, A, B) \
    case N: return Spec<Cx, A, B>::rows_fwd(P, refP, T, g, st);
        CPPHF_SPEC_SIZES(X)
#undef X
        default: break;
    }
    FftPlan1D pl;
    if (!make_plan(g.n1, pl)) return fail(CPPHF_ERR_INVALID, "exchange: mesh size has too many prime factors");
    Gen<Cx>::attrs();
    const Launch L = plan_launch(g.n1, g.C, sizeof(Cx), g.n1, true);
    if (L.smem > kSmemMax) return fail(CPPHF_ERR_UNSUPPORTED, "exchange: mesh axis too long for the shared-memory FFT");
    k_rows_fwd_g<Cx><<<dim3(g.n0, L.nchunk), cap_threads(k_rows_fwd_g<Cx>, L.threads), L.smem, st>>>(P, refP, T, g,
                                                                                                     pl, L.CB);
    CPPHF_LAUNCH_CHECK("exchange rows forward");
    return CPPHF_OK;
}

template <class Cx>
int pass_cols(Cx* T, const double2* VR, const ExchangeGeom& g, int vmode, cudaStream_t st) {
    switch (g.n0) {
#define X(N, A, B) \
    case N: return Spec<Cx, A, B>::cols(T, VR, g, vmode, st);
        CPPHF_SPEC_SIZES(X)
#undef X
        default: break;
    }
    FftPlan1D pl;
    if (!make_plan(g.n0, pl)) return fail(CPPHF_ERR_INVALID, "exchange: mesh size has too many prime factors");
    Gen<Cx>::attrs();
    const Launch L = plan_launch(g.n0, g.C, sizeof(Cx), g.n0, true);
    if (L.smem > kSmemMax) return fail(CPPHF_ERR_UNSUPPORTED, "exchange: mesh axis too long for the shared-memory FFT");
    k_cols_conv_g<Cx><<<dim3(g.n1, L.nchunk), cap_threads(k_cols_conv_g<Cx>, L.threads), L.smem, st>>>(T, VR, g, pl,
                                                                                                       L.CB, vmode);
    CPPHF_LAUNCH_CHECK("exchange columns convolve");
    return CPPHF_OK;
}

template <class Cx>
int pass_rows_inv(const Cx* T, double2* Sigma, const ExchangeGeom& g, double scale, cudaStream_t st) {
    switch (g.n1) {
#define X(N, A, B) \
    case N: return Spec<Cx, A, B>::rows_inv(T, Sigma, g, scale, st);
        CPPHF_SPEC_SIZES(X)
#undef X
        default: break;
    }
    FftPlan1D pl;
    if (!make_plan(g.n1, pl)) return fail(CPPHF_ERR_INVALID, "exchange: mesh size has too many prime factors");
    Gen<Cx>::attrs();
    const Launch L = plan_launch(g.n1, g.C, sizeof(Cx), g.n1, true);
    if (L.smem > kSmemMax) return fail(CPPHF_ERR_UNSUPPORTED, "exchange: mesh axis too long for the shared-memory FFT");
    k_rows_inv_g<Cx><<<dim3(g.n0, L.nchunk), cap_threads(k_rows_inv_g<Cx>, L.threads), L.smem, st>>>(T, Sigma, g, pl,
                                                                                                     L.CB, scale);
    CPPHF_LAUNCH_CHECK("exchange rows inverse");
    return CPPHF_OK;
}

template <class Cx>
int launch_exchange(const double2* P, const double2* refP, const double2* VR, double2* Sigma, Cx* T,
                    const ExchangeGeom& g, cudaStream_t st, int vmode = kColsVR) {
    CPPHF_TRY(pass_rows_fwd<Cx>(P, refP, T, g, st));
    CPPHF_TRY(pass_cols<Cx>(T, VR, g, vmode, st));
    CPPHF_TRY(pass_rows_inv<Cx>(T, Sigma, g, -1.0 / ((double)g.n0 * (double)g.n1), st));
    return CPPHF_OK;
}

}  // namespace

namespace {

// bytes of the intermediate T the launch needs (0: T aliases Sigma)
size_t exchange_t_bytes(int64_t nk1, int64_t nk2, int64_t nb, int hcp, int precision) {
    const size_t nk = (size_t)nk1 * nk2;
    const size_t C = hcp ? (size_t)nb * (nb + 1) / 2 : (size_t)nb * nb;
    if (precision == 32) return (nk * C * sizeof(float2) + 255) & ~(size_t)255;
    if (hcp) return (nk * C * sizeof(double2) + 255) & ~(size_t)255;
    return 0;
}

}  // namespace

// T when it does not alias Sigma (0 for the full FP64 form).
size_t exchange_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb, int hcp, int precision) {
    return exchange_t_bytes(nk1, nk2, nb, hcp, precision);
}

int exchange_columns(void* T, const double2* VR, const ExchangeGeom& g, int precision, cudaStream_t st) {
    if (precision == 32) return pass_cols<float2>(static_cast<float2*>(T), VR, g, kColsVR, st);
    return pass_cols<double2>(static_cast<double2*>(T), VR, g, kColsVR, st);
}

int exchange(const double2* P, const double2* refP, const double2* VR, double2* Sigma, int64_t nk1, int64_t nk2,
             int64_t nb, int64_t dv, int hcp, int shift, int precision, void* workspace, size_t workspace_bytes,
             cudaStream_t st) {
    if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(CPPHF_ERR_INVALID, "exchange: empty mesh or nb");
    if (nk1 > 65535 || nk2 > 65535 || nb > 4096) return fail(CPPHF_ERR_INVALID, "exchange: size out of range");
    if (!(dv == 1 || dv == nb)) return fail(CPPHF_ERR_INVALID, "VR shape must be (..., 1, 1) or (..., nb, nb).");
    if (hcp && dv != 1)
        return fail(CPPHF_ERR_INVALID, "hermitian_channel_packing requires VR with shape (...,1,1)");
    if (precision != 32 && precision != 64) return fail(CPPHF_ERR_INVALID, "exchange: precision must be 32 or 64");
    if (!P || !VR || !Sigma) return fail(CPPHF_ERR_INVALID, "exchange: null pointer");
    ExchangeGeom g;
    g.n0 = (int)nk1;
    g.n1 = (int)nk2;
    g.nb = (int)nb;
    g.hcp = hcp ? 1 : 0;
    g.C = hcp ? (int)(nb * (nb + 1) / 2) : (int)(nb * nb);
    g.dv = dv == 1 ? 1 : (int)(nb * nb);
    g.Ct = g.C;
    g.shift = shift ? 1 : 0;
    g.err = wait_error_word();
    if (!g.err) return CPPHF_ERR_CUDA;
    const size_t need = exchange_t_bytes(nk1, nk2, nb, hcp, precision);
    if (need > 0 && (workspace == nullptr || workspace_bytes < need))
        return fail(CPPHF_ERR_INVALID, "exchange: workspace too small (" +
                                           std::to_string(exchange_workspace_bytes(nk1, nk2, nb, hcp, precision)) +
                                           " bytes needed)");
    if (precision == 32)
        return launch_exchange<float2>(P, refP, VR, Sigma, static_cast<float2*>(workspace), g, st, kColsVR);
    double2* T = hcp ? static_cast<double2*>(workspace) : Sigma;
    return launch_exchange<double2>(P, refP, VR, Sigma, T, g, st, kColsVR);
}

namespace {

// dL/dVR = -(1/nk) conj(X^)(q) G^(q) per channel (dv = nb*nb) or summed over the
// channels (dv = 1); X^, G^ are the 2-D forward transforms, layout (q, C).
__global__ void k_vr_grad(const double2* __restrict__ Xh, const double2* __restrict__ Gh, double2* __restrict__ gVR,
                          int64_t nk, int C, int dv, double scale) {
    if (dv != 1) {
        const int64_t n = nk * C;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            gVR[i] = cscale(cmul(cconj(Xh[i]), Gh[i]), scale);
        return;
    }
    // one warp per q; fixed lane order -> deterministic
    const int lane = threadIdx.x & 31;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nk; q += warps) {
        double2 acc = mk(0.0, 0.0);
        for (int c = lane; c < C; c += 32) cfma(acc, cconj(Xh[q * C + c]), Gh[q * C + c]);
        acc.x = warp_sum(acc.x);
        acc.y = warp_sum(acc.y);
        if (lane == 0) gVR[q] = cscale(acc, scale);
    }
}

int check_adjoint_args(int64_t nk1, int64_t nk2, int64_t nb, int64_t dv) {
    if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(CPPHF_ERR_INVALID, "exchange: empty mesh or nb");
    if (nk1 > 65535 || nk2 > 65535 || nb > 4096) return fail(CPPHF_ERR_INVALID, "exchange: size out of range");
    if (!(dv == 1 || dv == nb)) return fail(CPPHF_ERR_INVALID, "VR shape must be (..., 1, 1) or (..., nb, nb).");
    return CPPHF_OK;
}

ExchangeGeom full_geom(int64_t nk1, int64_t nk2, int64_t nb, int64_t dv) {
    ExchangeGeom g;
    g.n0 = (int)nk1;
    g.n1 = (int)nk2;
    g.nb = (int)nb;
    g.hcp = 0;
    g.C = (int)(nb * nb);
    g.dv = dv == 1 ? 1 : (int)(nb * nb);
    g.Ct = g.C;
    g.shift = 0;
    g.err = wait_error_word();
    return g;
}

}  // namespace

int exchange_adjoint(const double2* G, const double2* VR, double2* gP, int64_t nk1, int64_t nk2, int64_t nb,
                     int64_t dv, cudaStream_t st) {
    CPPHF_TRY(check_adjoint_args(nk1, nk2, nb, dv));
    if (!G || !VR || !gP) return fail(CPPHF_ERR_INVALID, "exchange_adjoint: null pointer");
    const ExchangeGeom g = full_geom(nk1, nk2, nb, dv);
    return launch_exchange<double2>(G, nullptr, VR, gP, gP, g, st, kColsConjVR);
}

size_t exchange_vr_grad_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb) {
    return 2 * (size_t)nk1 * nk2 * nb * nb * sizeof(double2);
}

int exchange_vr_grad(const double2* P, const double2* refP, const double2* G, double2* gVR, int64_t nk1, int64_t nk2,
                     int64_t nb, int64_t dv, void* ws, size_t wsb, cudaStream_t st) {
    CPPHF_TRY(check_adjoint_args(nk1, nk2, nb, dv));
    if (!P || !G || !gVR) return fail(CPPHF_ERR_INVALID, "exchange_vr_grad: null pointer");
    const size_t need = exchange_vr_grad_workspace_bytes(nk1, nk2, nb);
    if (!ws || wsb < need)
        return fail(CPPHF_ERR_INVALID, "exchange_vr_grad: workspace too small (" + std::to_string(need) + " bytes needed)");
    const ExchangeGeom g = full_geom(nk1, nk2, nb, dv);
    double2* Xh = static_cast<double2*>(ws);
    double2* Gh = Xh + (size_t)nk1 * nk2 * g.C;
    CPPHF_TRY(pass_rows_fwd<double2>(P, refP, Xh, g, st));
    CPPHF_TRY(pass_cols<double2>(Xh, nullptr, g, kColsForwardOnly, st));
    CPPHF_TRY(pass_rows_fwd<double2>(G, nullptr, Gh, g, st));
    CPPHF_TRY(pass_cols<double2>(Gh, nullptr, g, kColsForwardOnly, st));
    const int64_t nk = nk1 * nk2;
    const int64_t work = dv == 1 ? nk * 32 : nk * g.C;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)num_sms() * 8));
    k_vr_grad<<<grid, 256, 0, st>>>(Xh, Gh, gVR, nk, g.C, g.dv, -1.0 / (double)nk);
    CPPHF_LAUNCH_CHECK("exchange VR gradient");
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

int cpphf_exchange_adjoint(const void* G, const void* VR, void* gP, int64_t nk1, int64_t nk2, int64_t nb, int64_t dv,
                           void* stream) {
    return cpphf::exchange_adjoint(static_cast<const double2*>(G), static_cast<const double2*>(VR),
                                   static_cast<double2*>(gP), nk1, nk2, nb, dv, static_cast<cudaStream_t>(stream));
}

size_t cpphf_exchange_vr_grad_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb) {
    return cpphf::exchange_vr_grad_workspace_bytes(nk1, nk2, nb);
}

int cpphf_exchange_vr_grad(const void* P, const void* refP, const void* G, void* gVR, int64_t nk1, int64_t nk2,
                           int64_t nb, int64_t dv, void* workspace, size_t workspace_bytes, void* stream) {
    return cpphf::exchange_vr_grad(static_cast<const double2*>(P), static_cast<const double2*>(refP),
                                   static_cast<const double2*>(G), static_cast<double2*>(gVR), nk1, nk2, nb, dv,
                                   workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

size_t cpphf_exchange_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb, int hcp, int precision) {
    return cpphf::exchange_workspace_bytes(nk1, nk2, nb, hcp, precision);
}

int cpphf_exchange(const void* P, const void* refP, const void* VR, void* Sigma, int64_t nk1, int64_t nk2,
                   int64_t nb, int64_t dv, int hcp, int apply_ifftshift, int precision, void* workspace,
                   size_t workspace_bytes, void* stream) {
    return cpphf::exchange(static_cast<const double2*>(P), static_cast<const double2*>(refP),
                           static_cast<const double2*>(VR), static_cast<double2*>(Sigma), nk1, nk2, nb, dv, hcp,
                           apply_ifftshift, precision, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

int cpphf_clear_fft_plan_cache(void) { return CPPHF_OK; }

}  // extern "C"
