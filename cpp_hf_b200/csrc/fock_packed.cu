// Hermitian-packed Fock build: the exchange of cpp_hf selfenergy.hpp:119-171
// (upper-triangle channel packing) generalised from a scalar V(q) to an
// orbital-resolved V(q) that is Hermitian at every q, with the assembly of
// fock.hpp:34-351 fused into the last FFT pass.
//
// When V_ba(q) = conj V_ab(q) for every q (VR_ba(R) = conj VR_ab(-R)) and the
// density is Hermitian, the exchange self-energy is Hermitian too:
// Sigma_ba = conj Sigma_ab.  The build then transforms the nb(nb+1)/2 channels
// a <= b only (36 of 64 at nb = 8), and the last pass writes F directly:
//   A  rows:    P[kx, :, upper-triangle row segments] (- refP), FFT along ky -> T
//   B  columns: FFT along kx, * VR (packed like T), IFFT along kx (exchange.cu)
//   C  rows:    IFFT along ky, * (-1/(nk1 nk2)) = Sigma_ab; then per element
//               F_ab = herm(h)_ab + Sigma_ab + herm(SC)_ab + delta_ab hd_a,
//               F_ba = conj F_ab, optional Sigma / dense H, and the energy
//               w_k m_ab Re[herm(h)_ab conj P_ab + Sigma_ab conj(P - refP)_ab / 2]
//               (m = 1 on the diagonal, 2 off it), Kahan-summed per thread,
//               reduced by the last block, which adds the k-independent terms
//               (Sigma_C + diag H)(rho_bar) / 2.
// T is a workspace field of nk x Ct packed channels that stays in L2 between
// the passes; P, h (its Hermitian part, packed once per kernel), VR (packed
// once per kernel) and F cross DRAM once per build (P twice: pass C reads
// its upper triangle again for the energy).
//
// Packed channel layout: chunk q (0 <= q < ceil(nb/2)) holds row r1 = q from
// its diagonal (L1 = nb - q channels) then row r2 = nb-1-q from its diagonal
// (L2 = q + 1 channels; none for the middle row of odd nb), nb + 1 channels
// per chunk, padded to an even number CBp of slots (so that the TMA x
// coordinate of a chunk is a multiple of 16 bytes for complex64 too; the same
// layout serves both precisions of a switched solve).
#include "bulk.cuh"
#include "common.cuh"
#include "exchange.cuh"
#include "exchange_pipe.cuh"
#include "fft_reg.cuh"
#include "fock.cuh"
#include "team.cuh"

#include <algorithm>
#include <mutex>
#include <string>

namespace cpphf {

namespace {

constexpr int kPackMaxNb = 8;
constexpr int kPackStages = 2;
constexpr int kPackMaxThreads = 256;

__host__ __device__ __forceinline__ void pack_rows(int nb, int q, int& r1, int& r2, int& L1, int& L2) {
    r1 = q;
    r2 = nb - 1 - q;
    L1 = nb - r1;
    L2 = (r2 > r1) ? nb - r2 : 0;
}

// Once per kernel: VRp[k, slot] = VR[k, r, j] (dv = nb) and
// hp[k, slot] = (h[k, r, j] + conj h[k, j, r]) / 2, zero in padding slots.
__global__ void k_pack_fields(const double2* __restrict__ VR, int dv, const double2* __restrict__ h,
                              double2* __restrict__ VRp, double2* __restrict__ hp, int64_t nk, PackGeom pg) {
    const int nb = pg.nb, nb2 = nb * nb;
    const int64_t n = nk * pg.Ct;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = idx / pg.Ct;
        const int s = (int)(idx - k * pg.Ct);
        const int q = s / pg.CBp, c = s - q * pg.CBp;
        int r1, r2, L1, L2;
        pack_rows(nb, q, r1, r2, L1, L2);
        double2 v = mk(0.0, 0.0), hv = mk(0.0, 0.0);
        if (c < L1 + L2) {
            const int r = c < L1 ? r1 : r2;
            const int j = c < L1 ? r1 + c : r2 + (c - L1);
            if (dv != 1) v = VR[(size_t)k * nb2 + r * nb + j];
            const double2 x = h[(size_t)k * nb2 + r * nb + j], y = h[(size_t)k * nb2 + j * nb + r];
            hv = mk(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
        }
        if (VRp) VRp[idx] = v;
        if (hp) hp[idx] = hv;
    }
}

// One tensor map per row-segment length L = 1..nb over a (n0, n1, nb*nb)
// complex128 field viewed as {2 nb^2 doubles, n1, n0}: box {2L, N, 1}.
struct SegMaps {
    CUtensorMap m[kPackMaxNb];
};

// &maps.m[L - 1] with compile-time indices only, so the address is always the
// kernel parameter's own (a tensor map must be read from parameter, constant
// or global memory, never from a local copy).
__device__ __forceinline__ const CUtensorMap* seg_map(const SegMaps& maps, int L) {
    switch (L) {
        case 1: return &maps.m[0];
        case 2: return &maps.m[1];
        case 3: return &maps.m[2];
        case 4: return &maps.m[3];
        case 5: return &maps.m[4];
        case 6: return &maps.m[5];
        case 7: return &maps.m[6];
        default: return &maps.m[7];
    }
}

// Pass A shared memory: tw[N] | mbar[kMaxPipeStages] | nst stages of
// { P segments, refP segments }, each array's two segments in seg_bytes (the
// second segment 128-byte aligned).
struct RowsPkLayout {
    size_t tw, bar, stage0, seg_bytes, stage_bytes, total;
};

__host__ __device__ inline RowsPkLayout rows_pk_layout(int N, int nb, bool ref, int nst) {
    RowsPkLayout L;
    L.tw = 0;
    L.bar = (sizeof(double2) * (size_t)N + 15) & ~(size_t)15;
    L.stage0 = (L.bar + 8 * kMaxPipeStages + 127) & ~(size_t)127;
    L.seg_bytes = (sizeof(double2) * (size_t)N * (nb + 1) + 128 + 127) & ~(size_t)127;
    L.stage_bytes = L.seg_bytes * (ref ? 2 : 1);
    L.total = L.stage0 + (size_t)nst * L.stage_bytes + 128;
    return L;
}

__host__ __device__ __forceinline__ size_t seg2_offset(int N, int L1) {
    return (sizeof(double2) * (size_t)N * L1 + 127) & ~(size_t)127;
}

// pass A: rows forward of the packed channels.  Tile t -> (kx = t / nchunk, chunk q).
// Thread (c, a): packed channel c of the chunk, line lane a.
template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(kPackMaxThreads, 2)
    k_rows_fwd_pk(const __grid_constant__ SegMaps mP, const __grid_constant__ SegMaps mR, int has_refP, Cx* T,
                  ExchangeGeom g, PackGeom pg, int ntiles, int nst) {
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    unsigned char* smem_raw = align128(smem_dyn);
    const bool has_ref = has_refP != 0;
    const int nb = pg.nb;
    const RowsPkLayout L = rows_pk_layout(N, nb, has_ref, nst);
    Cx* tw = reinterpret_cast<Cx*>(smem_raw + L.tw);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw + L.bar);
    const int c = threadIdx.x % pg.CB, a = threadIdx.x / pg.CB;
    build_line_twiddles(tw, N);
    if (threadIdx.x == 0) {
        for (int b = 0; b < nst; ++b) mbar_init(&bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int stage) {
        if (threadIdx.x != 0) return;
        const int kx = t / pg.nchunk, q = t - kx * pg.nchunk;
        int r1, r2, L1, L2;
        pack_rows(nb, q, r1, r2, L1, L2);
        const unsigned bytes = (unsigned)(sizeof(double2) * (size_t)N * (L1 + L2));
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        const size_t off2 = seg2_offset(N, L1);
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[stage], bytes * (has_ref ? 2u : 1u));
        tma_load_3d(st, seg_map(mP, L1), 2 * (r1 * nb + r1), 0, kx, &bar[stage]);
        if (L2) tma_load_3d(st + off2, seg_map(mP, L2), 2 * (r2 * nb + r2), 0, kx, &bar[stage]);
        if (has_ref) {
            tma_load_3d(st + L.seg_bytes, seg_map(mR, L1), 2 * (r1 * nb + r1), 0, kx, &bar[stage]);
            if (L2) tma_load_3d(st + L.seg_bytes + off2, seg_map(mR, L2), 2 * (r2 * nb + r2), 0, kx, &bar[stage]);
        }
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
        const int kx = t / pg.nchunk, q = t - kx * pg.nchunk;
        int r1, r2, L1, L2;
        pack_rows(nb, q, r1, r2, L1, L2);
        const bool live = c < L1 + L2;
        const bool first = c < L1;
        const int stride = first ? L1 : L2;
        const size_t base = first ? 0 : seg2_offset(N, L1);
        const int col = first ? c : c - L1;
        const double2* in = reinterpret_cast<const double2*>(st + base) + col;
        const double2* rin = reinterpret_cast<const double2*>(st + L.seg_bytes + base) + col;
        Cx v[N1];
        if (live && a < N2) {
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) {
                double2 x = in[(N2 * n1 + a) * stride];
                if (has_ref) x = csub(x, rin[(N2 * n1 + a) * stride]);
                v[n1] = to_c(x, Cx{});
            }
            dft<N1, false>(v);
        }
        __syncthreads();
        // in place: the channel's own column of its segment, now holding Cx values
        Cx* S = reinterpret_cast<Cx*>(st + base) + col;
        if (live && a < N2) {
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) S[(k1 * N2 + a) * stride] = cmul(v[k1], tw[a * k1]);
        }
        __syncthreads();
        if (live && a < N1) {
            Cx u[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) u[n2] = S[(a * N2 + n2) * stride];
            dft<N2, false>(u);
            const int ch = q * pg.CBp + c;
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) st_l2(T + ((size_t)kx * g.n1 + (a + N1 * k2)) * pg.Ct + ch, u[k2]);
        }
        __syncthreads();
    }
}

struct FusedOut {
    const double2* hp;       // packed Hermitian part of h (nk, Ct)
    const double2* P;        // density field
    const double2* refP;     // reference density field or null
    const double* w;         // per-k weights
    const double* hd;        // Hartree diagonal (nb) or null
    const double2* SC;       // contact self-energy (nb, nb) or null
    const double2* rho_bar;  // sum_k w_k (P - refP), needed when hd or SC is present
    double2* F;
    double2* Sigma;   // optional
    double2* Hdense;  // optional
    double* part;     // energy partials [gridDim.x]
    unsigned* counter;
    double* energy;   // optional
};

// k-independent energy terms: (1/2) Re sum_ij (SC_ij + delta_ij hd_i) rho_bar_ji
__device__ double kindep_energy(const FusedOut& o, int nb) {
    if (!o.rho_bar || (!o.hd && !o.SC)) return 0.0;
    double e = 0.0;
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            double2 x = o.SC ? o.SC[i * nb + j] : mk(0.0, 0.0);
            if (i == j && o.hd) x.x += o.hd[i];
            const double2 r = o.rho_bar[j * nb + i];
            e += 0.5 * (x.x * r.x - x.y * r.y);
        }
    return e;
}

// pass C: rows inverse of the packed channels with the Fock assembly and the
// energy fused in.  Tile t -> (kx = t / nchunk, chunk q).
template <class Cx, int N1, int N2>
__global__ void __launch_bounds__(kPackMaxThreads, 2)
    k_rows_inv_fock_pk(const __grid_constant__ CUtensorMap mT, FusedOut o, ExchangeGeom g, PackGeom pg, int ntiles,
                       double scale, int nst) {
    constexpr int N = N1 * N2;
    constexpr int kLanes = N1 > N2 ? N1 : N2;  // line lanes: blockDim.x = kLanes * CBp
    constexpr int NE = N / kLanes;             // epilogue points per thread (ky = a + kLanes e)
    constexpr int EB = 2;                      // epilogue points whose loads are issued together (4 and 6: more spills, slower)
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    __shared__ double red[32];
    unsigned char* smem_raw = align128(smem_dyn);
    const int CBp = pg.CBp, nb = pg.nb, nb2 = nb * nb;
    const PipeLayout L = pipe_layout(N, CBp, sizeof(Cx), false, nst);
    Cx* tw = reinterpret_cast<Cx*>(smem_raw + L.tw);
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw + L.bar);
    const int c = threadIdx.x % CBp, a = threadIdx.x / CBp;
    build_line_twiddles(tw, N);
    if (threadIdx.x == 0) {
        for (int b = 0; b < nst; ++b) mbar_init(&bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t, int stage) {
        if (threadIdx.x != 0) return;
        const int kx = t / pg.nchunk, q = t - kx * pg.nchunk;
        unsigned char* st = smem_raw + L.stage0 + (size_t)stage * L.stage_bytes;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[stage], (unsigned)(N * CBp * sizeof(Cx)));
        tma_load_3d(st, &mT, 2 * q * CBp, 0, kx, &bar[stage]);
    };
    Kahan e_k;
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
        Cx* S = reinterpret_cast<Cx*>(smem_raw + L.stage0 + (size_t)stage * L.stage_bytes);
        const int kx = t / pg.nchunk, q = t - kx * pg.nchunk;
        int r1, r2, L1, L2;
        pack_rows(nb, q, r1, r2, L1, L2);
        const bool live = c < L1 + L2;
        {
            Cx u[N2];
            if (live && a < N1) {
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) u[k2] = S[(a + N1 * k2) * CBp + c];
                dft<N2, true>(u);
            }
            __syncthreads();
            if (live && a < N1) {
#pragma unroll
                for (int na = 0; na < N2; ++na) S[(a * N2 + na) * CBp + c] = cmulc(u[na], tw[na * a]);
            }
        }
        __syncthreads();
        {
            Cx v[N1];
            if (live && a < N2) {
#pragma unroll
                for (int k1 = 0; k1 < N1; ++k1) v[k1] = S[(k1 * N2 + a) * CBp + c];
                dft<N1, true>(v);
            }
            __syncthreads();
            // the line back into the stage in natural ky order, then the epilogue
            // walks (ky, channel) with a short body (no register array live)
            if (live && a < N2) {
#pragma unroll
                for (int nbx = 0; nbx < N1; ++nbx) S[(a + N2 * nbx) * CBp + c] = v[nbx];
            }
        }
        __syncthreads();
        if (live) {
            const int r = c < L1 ? r1 : r2;
            const int jc = c < L1 ? r1 + c : r2 + (c - L1);
            const bool diag = r == jc;
            const int rj = r * nb + jc, jr = jc * nb + r;
            double2 sc_rj = mk(0.0, 0.0), sc_jr = mk(0.0, 0.0);
            if (o.SC) {
                sc_rj = o.SC[rj];
                sc_jr = o.SC[jr];
            }
            // Hermitian part of (SC + diag hd) at (r, jc)
            double2 add = mk(0.5 * (sc_rj.x + sc_jr.x), 0.5 * (sc_rj.y - sc_jr.y));
            const double hdr = (diag && o.hd) ? o.hd[r] : 0.0;
            add.x += hdr;
            const double mult = diag ? 1.0 : 2.0;
            const size_t slot = (size_t)q * CBp + c;
            // this thread's NE points ky = a + kLanes e, in batches of EB whose
            // loads are all issued before their first use (one memory latency
            // per batch instead of one per point)
#pragma unroll 1
            for (int e0 = 0; e0 < NE; e0 += EB) {
                double2 hh[EB], pv[EB], rv[EB];
#pragma unroll
                for (int e = 0; e < EB; ++e) {
                    if (e0 + e < NE) {
                        const size_t k = (size_t)kx * g.n1 + (a + kLanes * (e0 + e));
                        hh[e] = ld_stream(o.hp + k * pg.Ct + slot);
                        pv[e] = ld_stream(o.P + k * nb2 + rj);
                        rv[e] = o.refP ? ld_stream(o.refP + k * nb2 + rj) : mk(0.0, 0.0);
                    }
                }
#pragma unroll
                for (int e = 0; e < EB; ++e) {
                    if (e0 + e < NE) {
                        const int ky = a + kLanes * (e0 + e);
                        const size_t k = (size_t)kx * g.n1 + ky;
                        const size_t base = k * nb2;
                        const double2 sg = cscale(to_d(S[ky * CBp + c]), scale);
                        double2 f = cadd(cadd(hh[e], sg), add);
                        if (diag) f.y = 0.0;
                        o.F[base + rj] = f;
                        if (!diag) o.F[base + jr] = cconj(f);
                        if (o.Sigma) {
                            o.Sigma[base + rj] = cadd(sg, sc_rj);
                            if (!diag) o.Sigma[base + jr] = cadd(cconj(sg), sc_jr);
                        }
                        if (o.Hdense) {
                            o.Hdense[base + rj] = mk(hdr, 0.0);
                            if (!diag) o.Hdense[base + jr] = mk(0.0, 0.0);
                        }
                        const double2 p = pv[e];
                        const double2 rho = csub(p, rv[e]);
                        const double term = (hh[e].x * p.x + hh[e].y * p.y) + 0.5 * (sg.x * rho.x + sg.y * rho.y);
                        e_k.add(o.w[k] * mult * term);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (o.energy) {
        double e_acc[1] = {e_k.s};
        double out[1];
        if (reduce_last_block<1>(e_acc, o.part, o.counter, out, red) && threadIdx.x == 0)
            *o.energy = out[0] + kindep_energy(o, nb);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bool make_seg_maps(SegMaps* m, const void* base, int n0, int n1, int nb, int N) {
    const unsigned long long row = 2ull * nb * nb * sizeof(double);
    for (int L = 1; L <= kPackMaxNb; ++L) {
        const int Lc = std::min(L, nb);  // lengths above nb are never used; keep a valid box
        if (!make_tensor_map_3d(&m->m[L - 1], base, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2ull * nb * nb,
                                (unsigned long long)n1, (unsigned long long)n0, row, row * (unsigned long long)n1,
                                2u * (unsigned)Lc, (unsigned)N, 1u))
            return false;
    }
    return true;
}

template <class Cx, int N1, int N2>
struct PackSpec {
    static void attrs() {
        static std::once_flag once;
        std::call_once(once, [] {
            raise_smem(k_rows_fwd_pk<Cx, N1, N2>);
            raise_smem(k_rows_inv_fock_pk<Cx, N1, N2>);
        });
    }
    static int lanes() { return N1 > N2 ? N1 : N2; }
    template <class K>
    static int pgrid(K kern, int threads, size_t smem, int ntiles) {
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem);
        (void)cudaGetLastError();
        if (per < 1) per = 1;
        return std::max(1, std::min(ntiles, per * num_sms()));
    }
    static bool fits(const PackGeom& pg, bool ref) {
        if (lanes() * pg.CB > kPackMaxThreads || lanes() * pg.CBp > kPackMaxThreads) return false;
        if (rows_pk_layout(N1 * N2, pg.nb, ref, kPackStages).total > kSmemMax) return false;
        if (pipe_layout(N1 * N2, pg.CBp, sizeof(Cx), false, kPackStages).total > kSmemMax) return false;
        return true;
    }
    static int rows_fwd(const double2* P, const double2* refP, Cx* T, const ExchangeGeom& g, const PackGeom& pg,
                        cudaStream_t st) {
        attrs();
        SegMaps mP, mR;
        if (!make_seg_maps(&mP, P, g.n0, g.n1, pg.nb, N1 * N2) ||
            !make_seg_maps(&mR, refP ? refP : P, g.n0, g.n1, pg.nb, N1 * N2))
            return fail(CPPHF_ERR_CUDA, "packed Fock build: tensor map encoding failed");
        const RowsPkLayout L = rows_pk_layout(N1 * N2, pg.nb, refP != nullptr, kPackStages);
        const int threads = lanes() * pg.CB;
        const int nt = g.n0 * pg.nchunk;
        const int grid = pgrid(k_rows_fwd_pk<Cx, N1, N2>, threads, L.total, nt);
        k_rows_fwd_pk<Cx, N1, N2><<<grid, threads, L.total, st>>>(mP, mR, refP != nullptr, T, g, pg, nt, kPackStages);
        CPPHF_LAUNCH_CHECK("packed Fock build: rows forward");
        return CPPHF_OK;
    }
    static int rows_inv(const Cx* T, const FusedOut& o, const ExchangeGeom& g, const PackGeom& pg, cudaStream_t st) {
        attrs();
        CUtensorMap mT;
        const unsigned long long row = 2ull * pg.Ct * (sizeof(Cx) / 2);
        if (!make_tensor_map_3d(&mT, T, sizeof(Cx) == 16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                2ull * pg.Ct, (unsigned long long)g.n1, (unsigned long long)g.n0, row,
                                row * (unsigned long long)g.n1, 2u * (unsigned)pg.CBp, (unsigned)(N1 * N2), 1u))
            return fail(CPPHF_ERR_CUDA, "packed Fock build: tensor map encoding failed");
        const PipeLayout L = pipe_layout(N1 * N2, pg.CBp, sizeof(Cx), false, kPackStages);
        const int threads = lanes() * pg.CBp;
        const int nt = g.n0 * pg.nchunk;
        const int grid = std::min(pgrid(k_rows_inv_fock_pk<Cx, N1, N2>, threads, L.total, nt), kFockMaxPartials);
        if (o.energy) CPPHF_CUDA(cudaMemsetAsync(o.counter, 0, sizeof(unsigned), st));
        k_rows_inv_fock_pk<Cx, N1, N2><<<grid, threads, L.total, st>>>(mT, o, g, pg, nt,
                                                                       -1.0 / ((double)g.n0 * (double)g.n1),
                                                                       kPackStages);
        CPPHF_LAUNCH_CHECK("packed Fock build: rows inverse + assembly");
        return CPPHF_OK;
    }
};

// line length -> (N1, N2) of a register codelet with a pipelined pass (N <= 256)
bool spec_split(int n, int& n1, int& n2) {
    switch (n) {
#define X(N, A, B)          \
    case N:                 \
        n1 = A;             \
        n2 = B;             \
        return N <= 256;
        CPPHF_SPEC_SIZES(X)
#undef X
        default: return false;
    }
}

PackGeom pack_geom(int nb) {
    PackGeom pg;
    pg.nb = nb;
    pg.nchunk = (nb + 1) / 2;
    pg.CB = nb + 1;
    pg.CBp = (pg.CB + 1) & ~1;
    pg.Ct = pg.nchunk * pg.CBp;
    return pg;
}

template <class Cx>
bool rows_fits(int n1, const PackGeom& pg, bool ref) {
    switch (n1) {
#define X(N, A, B) \
    case N: if constexpr (N <= 256) return PackSpec<Cx, A, B>::fits(pg, ref); else return false;
        CPPHF_SPEC_SIZES(X)
#undef X
        default: return false;
    }
}

template <class Cx>
int rows_fwd_dispatch(const double2* P, const double2* refP, Cx* T, const ExchangeGeom& g, const PackGeom& pg,
                      cudaStream_t st) {
    switch (g.n1) {
#define X(N, A, B) \
    case N: if constexpr (N <= 256) return PackSpec<Cx, A, B>::rows_fwd(P, refP, T, g, pg, st); else break;
        CPPHF_SPEC_SIZES(X)
#undef X
        default: break;
    }
    return fail(CPPHF_ERR_UNSUPPORTED, "packed Fock build: mesh size without a pipelined codelet");
}

template <class Cx>
int rows_inv_dispatch(const Cx* T, const FusedOut& o, const ExchangeGeom& g, const PackGeom& pg, cudaStream_t st) {
    switch (g.n1) {
#define X(N, A, B) \
    case N: if constexpr (N <= 256) return PackSpec<Cx, A, B>::rows_inv(T, o, g, pg, st); else break;
        CPPHF_SPEC_SIZES(X)
#undef X
        default: break;
    }
    return fail(CPPHF_ERR_UNSUPPORTED, "packed Fock build: mesh size without a pipelined codelet");
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

bool packed_fock_eligible(const cpphf_kernel* K) {
    if (!K || !K->hermitian_packing || !K->include_exchange) return false;
    if (K->sl && (K->sl->fock_active || K->sl->hartree_active)) return false;
    if (K->nb < 1 || K->nb > kPackMaxNb || !(K->dv == 1 || K->dv == K->nb)) return false;
    if (K->nk1 > 65535 || K->nk2 > 65535) return false;
    int a, b;
    if (!spec_split((int)K->nk1, a, b) || !spec_split((int)K->nk2, a, b)) return false;
    const PackGeom pg = pack_geom((int)K->nb);
    const bool ref = K->has_refP != 0;
    return K->exchange_precision == 32 ? rows_fits<float2>((int)K->nk2, pg, ref)
                                       : rows_fits<double2>((int)K->nk2, pg, ref);
}

size_t packed_field_bytes(const cpphf_kernel* K) {
    if (!K || K->nb < 1 || K->nb > kPackMaxNb) return 0;
    const PackGeom pg = pack_geom((int)K->nb);
    return round256(sizeof(double2) * (size_t)K->nk1 * K->nk2 * pg.Ct);
}

size_t packed_fock_workspace_bytes(const cpphf_kernel* K) {
    if (!packed_fock_eligible(K)) return 0;
    const PackGeom pg = pack_geom((int)K->nb);
    const size_t nk = (size_t)K->nk1 * K->nk2;
    const size_t elem = K->exchange_precision == 32 ? sizeof(float2) : sizeof(double2);
    size_t b = round256(elem * nk * pg.Ct);                        // T
    if (!K->h_packed) b += packed_field_bytes(K);                  // hp
    if (!K->VR_packed && K->dv != 1) b += packed_field_bytes(K);   // VRp
    return b;
}

int pack_kernel_fields(const cpphf_kernel* K, double2* VRp, double2* hp, cudaStream_t st) {
    if (!K || K->nb < 1 || K->nb > kPackMaxNb) return fail(CPPHF_ERR_INVALID, "kernel_pack: nb must be 1..8");
    if (!K->h || (VRp && (!K->VR || K->dv != K->nb)))
        return fail(CPPHF_ERR_INVALID, "kernel_pack: needs h, and VR of width nb for VR_packed");
    const PackGeom pg = pack_geom((int)K->nb);
    const int64_t nk = K->nk1 * K->nk2;
    const int64_t n = nk * pg.Ct;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 16));
    k_pack_fields<<<grid, 256, 0, st>>>(static_cast<const double2*>(K->VR), (int)K->dv,
                                         static_cast<const double2*>(K->h), VRp, hp, nk, pg);
    CPPHF_LAUNCH_CHECK("kernel_pack");
    return CPPHF_OK;
}

size_t solver_pack_bytes(const cpphf_kernel* K) {
    cpphf_kernel K32 = *K;
    K32.exchange_precision = 32;
    if (!packed_fock_eligible(K) && !packed_fock_eligible(&K32)) return 0;
    size_t b = 0;
    if (!K->h_packed) b += packed_field_bytes(K);
    if (!K->VR_packed && K->dv != 1) b += packed_field_bytes(K);
    return b;
}

int solver_pack(const cpphf_kernel* K, cpphf_kernel* out, void* ws, cudaStream_t st) {
    *out = *K;
    if (solver_pack_bytes(K) == 0) return CPPHF_OK;
    unsigned char* W = static_cast<unsigned char*>(ws);
    double2* hp = nullptr;
    double2* vp = nullptr;
    if (!K->h_packed) {
        hp = reinterpret_cast<double2*>(W);
        W += packed_field_bytes(K);
        out->h_packed = hp;
    }
    if (!K->VR_packed && K->dv != 1) {
        vp = reinterpret_cast<double2*>(W);
        out->VR_packed = vp;
    }
    return pack_kernel_fields(K, vp, hp, st);
}

size_t fock_bytes_packed_kernel(const cpphf_kernel* K) {
    cpphf_kernel Kc = *K;
    static const double2 placeholder = {0.0, 0.0};  // sizing only: marks the packed fields as present
    if (solver_pack_bytes(K) > 0) {
        if (!Kc.h_packed) Kc.h_packed = &placeholder;
        if (!Kc.VR_packed && Kc.dv != 1) Kc.VR_packed = &placeholder;
    }
    return build_fock_workspace_bytes(&Kc);
}

int build_fock_packed(const cpphf_kernel* K, const double2* P, double2* Sigma, double2* F, const double* hd,
                      const double2* SC, const double2* rho_bar, double* energy, double2* Hdense, double* part,
                      unsigned* counter, void* ws, size_t wsb, cudaStream_t st) {
    const PackGeom pg = pack_geom((int)K->nb);
    const size_t nk = (size_t)K->nk1 * K->nk2;
    const bool c64 = K->exchange_precision == 32;
    if (wsb < packed_fock_workspace_bytes(K)) return fail(CPPHF_ERR_INVALID, "packed Fock build: workspace too small");
    unsigned char* W = static_cast<unsigned char*>(ws);
    size_t off = round256((c64 ? sizeof(float2) : sizeof(double2)) * nk * pg.Ct);
    void* T = W;
    const double2* hp = static_cast<const double2*>(K->h_packed);
    const double2* VRp = static_cast<const double2*>(K->VR_packed);
    double2* hp_ws = nullptr;
    double2* VRp_ws = nullptr;
    if (!hp) {
        hp_ws = reinterpret_cast<double2*>(W + off);
        off += packed_field_bytes(K);
    }
    if (!VRp && K->dv != 1) {
        VRp_ws = reinterpret_cast<double2*>(W + off);
        off += packed_field_bytes(K);
    }
    if (hp_ws || VRp_ws) CPPHF_TRY(pack_kernel_fields(K, VRp_ws, hp_ws, st));
    if (!hp) hp = hp_ws;
    if (!VRp && K->dv != 1) VRp = VRp_ws;
    ExchangeGeom g;
    g.n0 = (int)K->nk1;
    g.n1 = (int)K->nk2;
    g.nb = (int)K->nb;
    g.hcp = 0;
    g.shift = 0;
    g.C = pg.Ct;
    g.Ct = pg.Ct;
    g.dv = K->dv == 1 ? 1 : pg.Ct;
    g.err = wait_error_word();
    if (!g.err) return CPPHF_ERR_CUDA;
    const double2* refP = K->has_refP ? static_cast<const double2*>(K->refP) : nullptr;
    FusedOut o;
    o.hp = hp;
    o.P = P;
    o.refP = refP;
    o.w = K->w2d;
    o.hd = hd;
    o.SC = SC;
    o.rho_bar = rho_bar;
    o.F = F;
    o.Sigma = Sigma;
    o.Hdense = Hdense;
    o.part = part;
    o.counter = counter;
    o.energy = energy;
    const double2* VRcols = K->dv == 1 ? static_cast<const double2*>(K->VR) : VRp;
    if (c64) {
        float2* Tc = static_cast<float2*>(T);
        CPPHF_TRY(rows_fwd_dispatch<float2>(P, refP, Tc, g, pg, st));
        CPPHF_TRY(exchange_columns(Tc, VRcols, g, 32, st));
        return rows_inv_dispatch<float2>(Tc, o, g, pg, st);
    }
    double2* Td = static_cast<double2*>(T);
    CPPHF_TRY(rows_fwd_dispatch<double2>(P, refP, Td, g, pg, st));
    CPPHF_TRY(exchange_columns(Td, VRcols, g, 64, st));
    return rows_inv_dispatch<double2>(Td, o, g, pg, st);
}

}  // namespace cpphf

extern "C" {

size_t cpphf_kernel_packed_bytes(const cpphf_kernel* K) { return cpphf::packed_field_bytes(K); }

int cpphf_kernel_pack(const cpphf_kernel* K, void* VR_packed, void* h_packed, void* stream) {
    return cpphf::pack_kernel_fields(K, static_cast<double2*>(VR_packed), static_cast<double2*>(h_packed),
                                     static_cast<cudaStream_t>(stream));
}

}  // extern "C"
