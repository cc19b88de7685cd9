// Exchange self-energy  Sigma(k) = -IFFT2[ FFT2(P - refP) . VR ]  on a (nk1, nk2)
// mesh with nb*nb channel-interleaved orbital pairs (cpp_hf selfenergy.hpp:60-171).
//
// Three passes over an (nk1, nk2, C) intermediate T, each a grid of CTAs that
// owns one full FFT line for a block of CB consecutive channels:
//   A  rows:    load P[kx, :, chunk] (- refP), FFT along ky              -> T
//   B  columns: load T[:, ky, chunk], FFT along kx, * VR, IFFT along kx   -> T
//                (optional ifftshift of the kx axis applied on the store)
//   C  rows:    load T[kx, :, chunk], IFFT along ky, * (-1/(nk1 nk2))     -> Sigma
//                (optional ifftshift of ky; HCP unpack + conjugate mirror)
// For the full FP64 path T aliases Sigma (every CTA reads its whole tile
// before writing it), so the compulsory DRAM traffic is P + VR + Sigma and the
// intermediate round trips stay in L2 (P and VR are streamed with evict-first
// loads).  HCP (upper-triangle packing) and the complex64 form use a
// workspace field for T.
#include "common.cuh"
#include "fft.cuh"
#include "exchange.cuh"

#include <algorithm>
#include <mutex>
#include <string>

namespace cpphf {

namespace {

// channel -> (row, col) offsets for the HCP packing, built per CTA in smem.
__device__ __forceinline__ void hcp_pair(int ch, int nb, int& i, int& j) {
    int r = 0, c = ch;
    while (c >= nb - r) {
        c -= nb - r;
        ++r;
    }
    i = r;
    j = r + c;
}

struct Tile {
    int CB;       // channels per tile
    int threads;  // block size
    size_t smem;  // dynamic shared memory bytes
};

template <class Cx>
Tile pick_tile(const FftPlan1D& pl, int C) {
    const int n = pl.n;
    const int cbmax = std::max(1, std::min(C, (kEptMax * 256) / std::max(n, 1)));
    const int nch = (C + cbmax - 1) / cbmax;
    const int CB = (C + nch - 1) / nch;
    int threads = (n * CB + kEptMax - 1) / kEptMax;
    threads = ((threads + 31) / 32) * 32;
    threads = std::max(64, std::min(1024, threads));
    Tile t;
    t.CB = CB;
    t.threads = threads;
    t.smem = sizeof(Cx) * (size_t)n + sizeof(Cx) * (size_t)n * CB * (pl.generic ? 2 : 1) +
             sizeof(int) * 2 * (size_t)CB;
    return t;
}

// Dynamic smem layout: [tw n][buf n*CB][alt n*CB if generic][map 2*CB ints]
template <class Cx>
struct SmemView {
    Cx* tw;
    Cx* buf;
    Cx* alt;
    int* map;  // map[2c] = source offset within the nb*nb block, map[2c+1] = mirror (or -1)
    __device__ SmemView(unsigned char* base, const FftPlan1D& pl, int CB) {
        tw = reinterpret_cast<Cx*>(base);
        buf = tw + pl.n;
        alt = pl.generic ? buf + (size_t)pl.n * CB : nullptr;
        map = reinterpret_cast<int*>(buf + (size_t)pl.n * CB * (pl.generic ? 2 : 1));
    }
};

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

// Pass A: rows forward.
template <class Cx>
__global__ void k_rows_fwd(const double2* __restrict__ P, const double2* __restrict__ refP,
                           Cx* T, ExchangeGeom g, FftPlan1D pl, int CB) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemView<Cx> s(smem_raw, pl, CB);
    const int kx = blockIdx.x;
    const int chunk0 = blockIdx.y * CB;
    const int n = pl.n;  // == n1
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

// Pass B: columns forward, * VR, columns inverse (in place on T).
template <class Cx>
__global__ void k_cols_conv(Cx* T, const double2* __restrict__ VR, ExchangeGeom g, FftPlan1D pl,
                            int CB) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemView<Cx> s(smem_raw, pl, CB);
    const int ky = blockIdx.x;
    const int chunk0 = blockIdx.y * CB;
    const int n = pl.n;  // == n0
    build_twiddles(s.tw, n);
    __syncthreads();
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int nx = e / CB, c = e - nx * CB;
        const int ch = chunk0 + c;
        Cx v = mk((decltype(Cx{}.x))0, (decltype(Cx{}.x))0);
        if (ch < g.C) v = ld_l2(T + ((size_t)nx * g.n1 + ky) * g.Ct + ch);
        s.buf[e] = v;
    }
    __syncthreads();
    Cx* r = fft_tile<false>(s.buf, s.alt, s.tw, pl, CB);
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int nx = e / CB, c = e - nx * CB;
        const int ch = chunk0 + c;
        if (ch < g.C) {
            const size_t vi = ((size_t)nx * g.n1 + ky) * g.dv + (g.dv == 1 ? 0 : ch);
            const double2 w = ld_stream(VR + vi);
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

// Pass C: rows inverse, scale, unpack into Sigma.
template <class Cx>
__global__ void k_rows_inv(const Cx* T, double2* Sigma, ExchangeGeom g, FftPlan1D pl, int CB,
                           double scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemView<Cx> s(smem_raw, pl, CB);
    const int kx = blockIdx.x;
    const int chunk0 = blockIdx.y * CB;
    const int n = pl.n;  // == n1
    build_twiddles(s.tw, n);
    build_map(s.map, chunk0, CB, g.C, g.nb, g.hcp);
    __syncthreads();
    for (int e = threadIdx.x; e < n * CB; e += blockDim.x) {
        const int ny = e / CB, c = e - ny * CB;
        const int ch = chunk0 + c;
        Cx v = mk((decltype(Cx{}.x))0, (decltype(Cx{}.x))0);
        if (ch < g.C) v = ld_l2(T + ((size_t)kx * g.n1 + ny) * g.Ct + ch);
        s.buf[e] = v;
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

template <class Cx>
void set_smem_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        const int mx = 227 * 1024;
        cudaFuncSetAttribute(k_rows_fwd<Cx>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_cols_conv<Cx>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_rows_inv<Cx>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    });
}

template <class Cx>
int launch_exchange(const double2* P, const double2* refP, const double2* VR, double2* Sigma,
                    Cx* T, ExchangeGeom g, cudaStream_t st) {
    FftPlan1D prow, pcol;
    if (!make_plan(g.n1, prow) || !make_plan(g.n0, pcol))
        return fail(CPPHF_ERR_INVALID, "exchange: mesh size has too many prime factors");
    set_smem_attrs<Cx>();
    const Tile tr = pick_tile<Cx>(prow, g.C);
    const Tile tc = pick_tile<Cx>(pcol, g.C);
    const size_t smem_max = 227 * 1024;
    if (tr.smem > smem_max || tc.smem > smem_max || (size_t)g.n1 * tr.CB > (size_t)kEptMax * 1024 ||
        (size_t)g.n0 * tc.CB > (size_t)kEptMax * 1024)
        return fail(CPPHF_ERR_INVALID, "exchange: mesh axis too long for the shared-memory FFT");
    const int nchr = (g.C + tr.CB - 1) / tr.CB;
    const int nchc = (g.C + tc.CB - 1) / tc.CB;
    k_rows_fwd<Cx><<<dim3(g.n0, nchr), tr.threads, tr.smem, st>>>(P, refP, T, g, prow, tr.CB);
    CPPHF_LAUNCH_CHECK("exchange rows forward");
    k_cols_conv<Cx><<<dim3(g.n1, nchc), tc.threads, tc.smem, st>>>(T, VR, g, pcol, tc.CB);
    CPPHF_LAUNCH_CHECK("exchange columns convolve");
    const double scale = -1.0 / ((double)g.n0 * (double)g.n1);
    k_rows_inv<Cx><<<dim3(g.n0, nchr), tr.threads, tr.smem, st>>>(T, Sigma, g, prow, tr.CB, scale);
    CPPHF_LAUNCH_CHECK("exchange rows inverse");
    return CPPHF_OK;
}

}  // namespace

size_t exchange_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb, int hcp, int precision) {
    const size_t nk = (size_t)nk1 * nk2;
    const size_t C = hcp ? (size_t)nb * (nb + 1) / 2 : (size_t)nb * nb;
    if (precision == 32) return nk * C * sizeof(float2);
    if (hcp) return nk * C * sizeof(double2);
    return 0;
}

int exchange(const double2* P, const double2* refP, const double2* VR, double2* Sigma, int64_t nk1,
             int64_t nk2, int64_t nb, int64_t dv, int hcp, int shift, int precision,
             void* workspace, size_t workspace_bytes, cudaStream_t st) {
    if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(CPPHF_ERR_INVALID, "exchange: empty mesh or nb");
    if (nk1 > (1 << 20) || nk2 > (1 << 20) || nb > 4096)
        return fail(CPPHF_ERR_INVALID, "exchange: size out of range");
    if (!(dv == 1 || dv == nb))
        return fail(CPPHF_ERR_INVALID, "VR shape must be (..., 1, 1) or (..., nb, nb).");
    if (hcp && dv != 1)
        return fail(CPPHF_ERR_INVALID, "hermitian_channel_packing requires VR with shape (...,1,1)");
    if (precision != 32 && precision != 64)
        return fail(CPPHF_ERR_INVALID, "exchange: precision must be 32 or 64");
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
    const size_t need = exchange_workspace_bytes(nk1, nk2, nb, hcp, precision);
    if (need > 0 && (workspace == nullptr || workspace_bytes < need))
        return fail(CPPHF_ERR_INVALID, "exchange: workspace too small (" + std::to_string(need) +
                                           " bytes needed)");
    if (precision == 32)
        return launch_exchange<float2>(P, refP, VR, Sigma, reinterpret_cast<float2*>(workspace), g,
                                       st);
    double2* T = hcp ? reinterpret_cast<double2*>(workspace) : Sigma;
    return launch_exchange<double2>(P, refP, VR, Sigma, T, g, st);
}

}  // namespace cpphf

extern "C" {

size_t cpphf_exchange_workspace_bytes(int64_t nk1, int64_t nk2, int64_t nb, int hcp,
                                      int precision) {
    return cpphf::exchange_workspace_bytes(nk1, nk2, nb, hcp, precision);
}

int cpphf_exchange(const void* P, const void* refP, const void* VR, void* Sigma, int64_t nk1,
                   int64_t nk2, int64_t nb, int64_t dv, int hcp, int apply_ifftshift,
                   int precision, void* workspace, size_t workspace_bytes, void* stream) {
    return cpphf::exchange(static_cast<const double2*>(P), static_cast<const double2*>(refP),
                           static_cast<const double2*>(VR), static_cast<double2*>(Sigma), nk1,
                           nk2, nb, dv, hcp, apply_ifftshift, precision, workspace,
                           workspace_bytes, static_cast<cudaStream_t>(stream));
}

int cpphf_clear_fft_plan_cache(void) { return CPPHF_OK; }

}  // extern "C"
