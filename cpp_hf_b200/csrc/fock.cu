// Fock assembly and Hartree-Fock energy (cpp_hf fock.hpp:34-383).
//
//   pre      (only with Hartree or contact terms): rho_bar = sum_k w_k (P - refP)
//            by per-block partials + fixed-order final sum; then
//            hartree_diag = HH n_vec (n_vec = Re diag rho_bar) and the contact
//            self-energy SC = sum_t g_t [Oi tr(Oj rho_bar) - Oi rho_bar Oj].
//   exchange Sigma = -IFFT2[FFT2(P - refP) VR] (exchange.cu), or zero.
//   assemble one thread per (k, i<=j) pair: Sigma += SC,
//            F = herm(h + Sigma + diag(hartree_diag)), energy partials
//            w_k Re[h_ij P_ji + (Sigma_ij + H_ij)/2 (P - refP)_ji] (+ the
//            mirrored term); optional dense H.
//   energy   Kahan-compensated per-thread sums, then fixed-order block and
//            grid trees (deterministic for a given grid).
#include "bulk.cuh"
#include "common.cuh"
#include "exchange.cuh"
#include "fock.cuh"
#include "superlattice.cuh"
#include "team.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>

namespace cpphf {

namespace {

constexpr int kAsmThreads = 256;
constexpr int kRedThreads = 256;
constexpr int kMaxPartials = kFockMaxPartials;
constexpr int kAsmMaxStages = 4;
constexpr int kTileElems = 1024;  // k-blocks of at most this many elements take the bulk-pipelined assembly

// rho_bar partials: grid (Gk, ceil(nb2 / CH)), CH channels per block, lanes =
// blockDim / CH k-lanes.
__global__ void k_rho_bar_partial(const double2* __restrict__ P, const double2* __restrict__ refP,
                                  const double* __restrict__ w, int64_t nk, int nb2, int CH,
                                  double2* __restrict__ part) {
    __shared__ double2 acc_sh[kRedThreads];
    const int lanes = blockDim.x / CH;
    const int c_local = threadIdx.x % CH, lane = threadIdx.x / CH;
    const int c = blockIdx.y * CH + c_local;
    const int Gk = gridDim.x;
    const int64_t per = (nk + Gk - 1) / Gk;
    const int64_t k0 = (int64_t)blockIdx.x * per, k1 = min(nk, k0 + per);
    double2 acc = mk(0.0, 0.0);
    if (lane < lanes && c < nb2) {
        for (int64_t k = k0 + lane; k < k1; k += lanes) {
            double2 v = P[(size_t)k * nb2 + c];
            if (refP) v = csub(v, refP[(size_t)k * nb2 + c]);
            const double wk = w[k];
            acc.x += wk * v.x;
            acc.y += wk * v.y;
        }
    }
    acc_sh[threadIdx.x] = acc;
    __syncthreads();
    if (lane == 0 && c < nb2) {
        double2 s = acc;
        for (int l = 1; l < lanes; ++l) s = cadd(s, acc_sh[l * CH + c_local]);
        part[(size_t)blockIdx.x * nb2 + c] = s;
    }
}

// Final: rho_bar, hartree_diag and the contact self-energy SC (single block).
__global__ void k_hartree_contact(const double2* __restrict__ part, int Gk, int nb,
                                  const double* __restrict__ HH, int include_hartree,
                                  int has_contact, int n_contact, const double* __restrict__ cg,
                                  const double2* __restrict__ Oi, const double2* __restrict__ Oj,
                                  double2* __restrict__ rho_bar, double* __restrict__ hd,
                                  double2* __restrict__ SC) {
    const int nb2 = nb * nb;
    for (int c = threadIdx.x; c < nb2; c += blockDim.x) {
        double2 s = mk(0.0, 0.0);
        for (int b = 0; b < Gk; ++b) s = cadd(s, part[(size_t)b * nb2 + c]);
        rho_bar[c] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        double s = 0.0;
        if (include_hartree)
            for (int j = 0; j < nb; ++j) s += HH[i * nb + j] * rho_bar[j * nb + j].x;
        hd[i] = s;
    }
    if (!has_contact) return;
    // SC_ij = sum_t g [Oi_ij tr(Oj rho) - (Oi rho Oj)_ij]
    __shared__ double2 tr_sh[64];
    for (int c = threadIdx.x; c < nb2; c += blockDim.x) SC[c] = mk(0.0, 0.0);
    __syncthreads();
    for (int t = 0; t < n_contact; ++t) {
        const double g = cg[t];
        if (g == 0.0) continue;
        const double2* oi = Oi + (size_t)t * nb2;
        const double2* oj = Oj + (size_t)t * nb2;
        if (threadIdx.x == 0) {
            double2 tr = mk(0.0, 0.0);
            for (int i = 0; i < nb; ++i)
                for (int j = 0; j < nb; ++j) tr = cadd(tr, cmul(oj[i * nb + j], rho_bar[j * nb + i]));
            tr_sh[0] = tr;
        }
        __syncthreads();
        const double2 tr = tr_sh[0];
        for (int c = threadIdx.x; c < nb2; c += blockDim.x) {
            const int i = c / nb, j = c - i * nb;
            // herm = Oi * tr * g ; fk = -g * (Oi rho Oj)
            const double2 herm = cscale(cmul(oi[c], tr), g);
            double2 orho_oj = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) {
                double2 orho = mk(0.0, 0.0);
                for (int m = 0; m < nb; ++m) orho = cadd(orho, cmul(oi[i * nb + m], rho_bar[m * nb + l]));
                orho_oj = cadd(orho_oj, cmul(orho, oj[l * nb + j]));
            }
            const double2 fk = cscale(orho_oj, -g);
            SC[c] = cadd(SC[c], cadd(herm, fk));
        }
        __syncthreads();
    }
}

struct AsmArgs {
    const double2* h;
    double2* Sigma;
    double2* F;
    const double2* P;
    const double2* refP;
    const double* w;
    const double* hd;     // may be null (no Hartree)
    const double2* SC;    // may be null (no contact)
    double2* Hdense;      // may be null
    int64_t nk;
    int nb;
    double* part;         // energy partials [gridDim.x]
    unsigned* err;        // device error word (bounded waits)
};

__global__ void __launch_bounds__(kAsmThreads) k_assemble(AsmArgs a) {
    __shared__ double red[64];
    const int nb = a.nb;
    const int npair = nb * (nb + 1) / 2;
    const int64_t total = a.nk * npair;
    Kahan e_k;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t / npair;
        int r = (int)(t - k * npair);
        int i = 0;
        while (r >= nb - i) {
            r -= nb - i;
            ++i;
        }
        const int j = i + r;
        const size_t base = (size_t)k * nb * nb;
        const size_t ij = base + (size_t)i * nb + j, ji = base + (size_t)j * nb + i;
        double2 sij = a.Sigma[ij], sji = a.Sigma[ji];
        if (a.SC) {
            sij = cadd(sij, a.SC[i * nb + j]);
            sji = cadd(sji, a.SC[j * nb + i]);
            a.Sigma[ij] = sij;
            if (i != j) a.Sigma[ji] = sji;
        }
        const double2 hij = a.h[ij], hji = a.h[ji];
        double2 Aij = cadd(hij, sij), Aji = cadd(hji, sji);
        const double hdi = a.hd ? a.hd[i] : 0.0;
        if (i == j) {
            Aij.x += hdi;
            Aji = Aij;
        }
        const double2 f = mk(0.5 * (Aij.x + Aji.x), 0.5 * (Aij.y - Aji.y));
        a.F[ij] = f;
        if (i != j) a.F[ji] = cconj(f);
        if (a.Hdense) {
            a.Hdense[ij] = mk(i == j ? hdi : 0.0, 0.0);
            if (i != j) a.Hdense[ji] = mk(0.0, 0.0);
        }
        // energy: w_k [Re(h_ij P_ji) + Re(inter_ij dP_ji)] (+ mirrored (j,i))
        const double2 pji = a.P[ji], pij = a.P[ij];
        double2 dji = pji, dij = pij;
        if (a.refP) {
            dji = csub(pji, a.refP[ji]);
            dij = csub(pij, a.refP[ij]);
        }
        double2 iij = cscale(sij, 0.5);
        if (i == j && a.hd) iij.x += 0.5 * hdi;
        double s = (hij.x * pji.x - hij.y * pji.y) + (iij.x * dji.x - iij.y * dji.y);
        if (i != j) {
            const double2 iji = cscale(sji, 0.5);
            s += (hji.x * pij.x - hji.y * pij.y) + (iji.x * dij.x - iji.y * dij.y);
        }
        e_k.add(a.w[k] * s);
    }
    double e_acc[1] = {e_k.s};
    block_sum<1>(e_acc, red);
    if (threadIdx.x == 0) a.part[blockIdx.x] = e_acc[0];
}


// Pipelined assembly: persistent CTAs walk tiles of KT whole k-blocks; thread
// 0 brings the NEXT tile's Sigma, h, P (and refP) segments into the other
// shared-memory stage with three (four) bulk copies while the CTA assembles the
// current one, so each SM keeps two tiles of loads in flight.  The energy is
// reduced in the same launch (last-block sum in a fixed order).
template <bool REF, int NBC>
__global__ void __launch_bounds__(kAsmThreads) k_assemble_bulk(AsmArgs a, int KT, int64_t ntiles,
                                                               unsigned* counter, double* energy_out, int nst) {
    constexpr int NARR = REF ? 4 : 3;
    extern __shared__ __align__(16) unsigned char smem_dyn[];
    __shared__ double red[32];
    __shared__ __align__(8) unsigned long long bar[kAsmMaxStages];
    const int nb = NBC > 0 ? NBC : a.nb, nb2 = nb * nb;
    const int tile = KT * nb2;
    double2* stg = reinterpret_cast<double2*>(
        (reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~(uintptr_t)127);
    if (threadIdx.x == 0) {
        for (int b = 0; b < nst; ++b) mbar_init(&bar[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int64_t t, int s) {
        if (threadIdx.x != 0) return;
        const int64_t k0 = t * KT;
        const int nkt = (int)((a.nk - k0) < (int64_t)KT ? (a.nk - k0) : (int64_t)KT);
        const unsigned bytes = (unsigned)(sizeof(double2) * (size_t)nkt * nb2);
        const size_t off = (size_t)k0 * nb2;
        double2* d = stg + (size_t)s * NARR * tile;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&bar[s], bytes * NARR);
        bulk_g2s(d, a.Sigma + off, bytes, &bar[s]);
        bulk_g2s(d + tile, a.h + off, bytes, &bar[s]);
        bulk_g2s(d + 2 * tile, a.P + off, bytes, &bar[s]);
        if (REF) bulk_g2s(d + 3 * tile, a.refP + off, bytes, &bar[s]);
    };
    Kahan e_k;
    int i = 0;
    for (int j = 0; j < nst - 1; ++j)
        if ((int64_t)blockIdx.x + (int64_t)j * gridDim.x < ntiles) issue(blockIdx.x + (int64_t)j * gridDim.x, j);
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
        const int s = i % nst;
        if (t + (int64_t)(nst - 1) * gridDim.x < ntiles) issue(t + (int64_t)(nst - 1) * gridDim.x, (i + nst - 1) % nst);
        if (!mbar_wait(&bar[s], (unsigned)((i / nst) & 1), a.err)) return;
        const double2* sS = stg + (size_t)s * NARR * tile;
        const double2* sH = sS + tile;
        const double2* sP = sS + 2 * tile;
        const double2* sR = sS + 3 * tile;
        const int64_t k0 = t * KT;
        const int nkt = (int)((a.nk - k0) < (int64_t)KT ? (a.nk - k0) : (int64_t)KT);
        const int n = nkt * nb2;
        const size_t base = (size_t)k0 * nb2;
        for (int es = threadIdx.x; es < n; es += blockDim.x) {
            // skewed order inside each k-block: slot (q, j) is element (q + j mod nb, j),
            // so 8 consecutive threads touch 8 different 16-byte bank groups both in
            // the element and in its transpose (row-major order puts the transposed
            // reads 128 bytes apart: an 8-way bank conflict)
            const int kl = es / nb2, sl = es - kl * nb2;
            const int q = sl / nb, j = sl - q * nb;
            const int ii = (q + j) < nb ? q + j : q + j - nb;
            const int r = ii * nb + j;
            const int e = kl * nb2 + r;
            const int eT = kl * nb2 + j * nb + ii;
            const double hdi = a.hd ? a.hd[ii] : 0.0;
            double2 se = sS[e], sT = sS[eT];
            if (a.SC) {
                se = cadd(se, a.SC[r]);
                sT = cadd(sT, a.SC[j * nb + ii]);
            }
            double2 Aij = cadd(sH[e], se);
            double2 Aji = cadd(sH[eT], sT);
            if (ii == j) {
                Aij.x += hdi;
                Aji = Aij;
            }
            a.F[base + e] = mk(0.5 * (Aij.x + Aji.x), 0.5 * (Aij.y - Aji.y));
            if (a.SC) a.Sigma[base + e] = se;
            if (a.Hdense) a.Hdense[base + e] = mk(ii == j ? hdi : 0.0, 0.0);
            const double2 pji = sP[eT];
            const double2 dji = REF ? csub(pji, sR[eT]) : pji;
            double2 inter = cscale(se, 0.5);
            if (ii == j && a.hd) inter.x += 0.5 * hdi;
            const double2 hv = sH[e];
            const double sv = (hv.x * pji.x - hv.y * pji.y) + (inter.x * dji.x - inter.y * dji.y);
            e_k.add(a.w[k0 + kl] * sv);
        }
        __syncthreads();
    }
    if (energy_out) {
        double e_acc[1] = {e_k.s};
        double out[1];
        if (reduce_last_block<1>(e_acc, a.part, counter, out, red) && threadIdx.x == 0) *energy_out = out[0];
    }
}

// Fixed-order sum of block partials by one warp (lane-strided, then a
// shuffle tree): deterministic for a given partial count.
__global__ void k_sum_partials(const double* __restrict__ part, int n, double* __restrict__ out) {
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += 32) s += part[b];
    s = warp_sum(s);
    if (threadIdx.x == 0) *out = s;
}

struct FockWs {
    size_t off_part, off_counter, off_rho_part, off_rho_bar, off_sc, off_hd, off_exch, off_pack, total;
    size_t off_sl, sl_bytes, off_slh, off_rho;
    int Gasm, Gk;
};

bool sl_fock(const cpphf_kernel* K) { return K->sl && K->sl->fock_active && K->include_exchange; }
bool sl_hart(const cpphf_kernel* K) { return K->sl && K->sl->hartree_active && K->include_hartree; }

// Bulk assembly shape: complex elements per array per stage (halved with
// refP) and stage count; 512 x 2 was the fastest of the shapes swept on the
// 192x192, nb = 8 workload.
struct AsmCfg {
    int elems;
    int nst;
};
constexpr AsmCfg kAsmCfg{512, 2};

FockWs fock_ws_layout(const cpphf_kernel* K) {
    FockWs L;
    const int64_t nk = K->nk1 * K->nk2;
    const int64_t nb = K->nb, nb2 = nb * nb;
    const int64_t npair = nb * (nb + 1) / 2;
    const int64_t need = (nk * npair + kAsmThreads - 1) / kAsmThreads;
    L.Gasm = (int)std::max<int64_t>(1, std::min<int64_t>(need, std::min(kMaxPartials, 8 * num_sms())));
    L.Gk = (int)std::max<int64_t>(1, std::min<int64_t>(nk, 2 * num_sms()));
    size_t o = 0;
    auto take = [&](size_t bytes) {
        size_t at = o;
        o += (bytes + 255) & ~(size_t)255;
        return at;
    };
    L.off_part = take(sizeof(double) * kMaxPartials);
    L.off_counter = take(sizeof(unsigned));
    L.off_rho_part = take(sizeof(double2) * (size_t)L.Gk * nb2);
    L.off_rho_bar = take(sizeof(double2) * nb2);
    L.off_sc = take(sizeof(double2) * nb2);
    L.off_hd = take(sizeof(double) * nb);
    const int hcp = (K->exchange_hcp && K->dv == 1) ? 1 : 0;
    L.off_exch = take(exchange_workspace_bytes(K->nk1, K->nk2, K->nb, hcp, K->exchange_precision));
    L.off_pack = take(packed_fock_workspace_bytes(K));
    L.sl_bytes = 0;
    L.off_sl = L.off_slh = L.off_rho = o;
    if (sl_fock(K)) {
        const cpphf_superlattice* sl = K->sl;
        L.sl_bytes = superlattice_workspace_bytes(sl->pair_start[sl->n_delta], sl->n_G, sl->dim_orb, sl->N_ext_x,
                                                  sl->N_ext_y, sl->V_lag_fft_orbital != nullptr);
        L.off_sl = take(L.sl_bytes);
        if (K->has_refP) L.off_rho = take(sizeof(double2) * (size_t)nk * nb2);
    }
    if (sl_hart(K)) L.off_slh = take(sl_hartree_workspace_bytes(K->sl));
    L.total = o;
    return L;
}

}  // namespace

int validate_kernel(const cpphf_kernel* K) {
    if (!K) return fail(CPPHF_ERR_INVALID, "kernel: null");
    if (K->nk1 < 1 || K->nk2 < 1 || K->nb < 1) return fail(CPPHF_ERR_INVALID, "h must be (nk1,nk2,nb,nb)");
    if (!(K->dv == 1 || K->dv == K->nb)) return fail(CPPHF_ERR_INVALID, "VR last two dims must be (1,1) or (nb,nb)");
    if (!K->h || !K->w2d) return fail(CPPHF_ERR_INVALID, "kernel: null h or w2d");
    if (K->include_exchange && !K->VR) return fail(CPPHF_ERR_INVALID, "kernel: null VR");
    if (K->has_refP && !K->refP) return fail(CPPHF_ERR_INVALID, "refP must match h shape when has_refP is true");
    if (K->include_hartree && !K->HH) return fail(CPPHF_ERR_INVALID, "kernel: null HH");
    if (K->has_contact && (!K->contact_g || !K->contact_Oi || !K->contact_Oj || K->n_contact < 1))
        return fail(CPPHF_ERR_INVALID, "kernel: contact arrays missing");
    if (K->has_contact && K->nb > 64) return fail(CPPHF_ERR_UNSUPPORTED, "contact terms need nb <= 64");
    if (K->exchange_precision != 32 && K->exchange_precision != 64)
        return fail(CPPHF_ERR_INVALID, "kernel: exchange_precision must be 32 or 64");
    if (K->sl && (K->sl->fock_active || K->sl->hartree_active)) {
        const cpphf_superlattice* sl = K->sl;
        if (sl->n_G < 1 || sl->dim_orb < 1 || sl->n_G * sl->dim_orb != K->nb)
            return fail(CPPHF_ERR_INVALID, "superlattice mode requires n_G × dim_orb == nb");
        if (sl->n_delta < 0 || !sl->pair_start || !sl->pair_to_delta || !sl->g_a_off)
            return fail(CPPHF_ERR_INVALID, "superlattice: missing layout arrays");
        if (sl->fock_active && (!sl->V_lag_fft || sl->N_ext_x < K->nk1 || sl->N_ext_y < K->nk2))
            return fail(CPPHF_ERR_INVALID, "V_lag_fft must have shape (N_ext_x, N_ext_y)");
        if (sl->hartree_active && K->include_hartree && !sl->HH_GG && !sl->HH_GG_orbital)
            return fail(CPPHF_ERR_INVALID, "HH_GG must be (n_G, n_G)");
    }
    return CPPHF_OK;
}

size_t build_fock_workspace_bytes(const cpphf_kernel* K) { return fock_ws_layout(K).total; }

int build_fock(const cpphf_kernel* K, const double2* P, double2* Sigma, double2* F, double* hd_out,
               double* energy, double2* Hdense, void* ws, size_t wsb, cudaStream_t st) {
    CPPHF_TRY(validate_kernel(K));
    if (!P || !F) return fail(CPPHF_ERR_INVALID, "build_fock: null pointer");
    const FockWs L = fock_ws_layout(K);
    if (!ws || wsb < L.total)
        return fail(CPPHF_ERR_INVALID, "build_fock: workspace too small (" + std::to_string(L.total) + " bytes needed)");
    unsigned char* W = static_cast<unsigned char*>(ws);
    double* part = reinterpret_cast<double*>(W + L.off_part);
    double2* rho_part = reinterpret_cast<double2*>(W + L.off_rho_part);
    double2* rho_bar = reinterpret_cast<double2*>(W + L.off_rho_bar);
    double2* SC = reinterpret_cast<double2*>(W + L.off_sc);
    double* hd = hd_out ? hd_out : reinterpret_cast<double*>(W + L.off_hd);
    const int64_t nk = K->nk1 * K->nk2;
    const int nb = (int)K->nb, nb2 = nb * nb;
    const double2* refP = K->has_refP ? static_cast<const double2*>(K->refP) : nullptr;
    const bool need_pre = K->include_hartree || K->has_contact;
    const bool slh = sl_hart(K);
    if (need_pre) {
        const int CH = std::min(nb2, kRedThreads);
        dim3 grid(L.Gk, (nb2 + CH - 1) / CH);
        k_rho_bar_partial<<<grid, kRedThreads, 0, st>>>(P, refP, K->w2d, nk, nb2, CH, rho_part);
        CPPHF_LAUNCH_CHECK("rho_bar partial");
        // the superlattice Hartree replaces the diagonal Hartree (fock.hpp:66-175)
        k_hartree_contact<<<1, 256, 0, st>>>(rho_part, L.Gk, nb, K->HH, K->include_hartree && !slh,
                                             K->has_contact, K->n_contact, K->contact_g,
                                             static_cast<const double2*>(K->contact_Oi),
                                             static_cast<const double2*>(K->contact_Oj), rho_bar,
                                             hd, SC);
        CPPHF_LAUNCH_CHECK("hartree/contact");
        if (slh) CPPHF_TRY(sl_hartree(K->sl, rho_bar, SC, K->has_contact, W + L.off_slh, st));
    } else if (hd_out) {
        CPPHF_CUDA(cudaMemsetAsync(hd, 0, sizeof(double) * nb, st));
    }
    if (packed_fock_eligible(K)) {
        unsigned* counter = reinterpret_cast<unsigned*>(W + L.off_counter);
        return build_fock_packed(K, P, Sigma, F, (K->include_hartree && !slh) ? hd : nullptr,
                                 (K->has_contact || slh) ? SC : nullptr, need_pre ? rho_bar : nullptr, energy,
                                 Hdense, part, counter, W + L.off_pack, wsb - L.off_pack, st);
    }
    if (!Sigma) return fail(CPPHF_ERR_INVALID, "build_fock: null Sigma");
    if (sl_fock(K)) {
        const cpphf_superlattice* sl = K->sl;
        const double2* rho = P;
        if (refP) {
            double2* tmp = reinterpret_cast<double2*>(W + L.off_rho);
            CPPHF_TRY(field_diff(P, refP, tmp, nk * nb2, st));
            rho = tmp;
        }
        CPPHF_TRY(superlattice_streamed(rho, static_cast<const double2*>(sl->V_lag_fft),
                                        static_cast<const double2*>(sl->V_lag_fft_orbital), sl->g_a_off, sl->pair_i,
                                        sl->pair_j, sl->pair_start, sl->n_delta, K->nk1, K->nk2, sl->n_G, sl->dim_orb,
                                        sl->N_ext_x, sl->N_ext_y, 1, Sigma, W + L.off_sl, L.sl_bytes, st));
    } else if (K->include_exchange) {
        const int hcp = (K->exchange_hcp && K->dv == 1) ? 1 : 0;
        CPPHF_TRY(exchange(P, refP, static_cast<const double2*>(K->VR), Sigma, K->nk1, K->nk2, K->nb,
                           K->dv, hcp, 0, K->exchange_precision, W + L.off_exch,
                           wsb - L.off_exch, st));
    } else {
        CPPHF_CUDA(cudaMemsetAsync(Sigma, 0, sizeof(double2) * (size_t)nk * nb2, st));
    }
    AsmArgs a;
    a.h = static_cast<const double2*>(K->h);
    a.Sigma = Sigma;
    a.F = F;
    a.P = P;
    a.refP = refP;
    a.w = K->w2d;
    a.hd = (K->include_hartree && !slh) ? hd : nullptr;
    a.SC = (K->has_contact || slh) ? SC : nullptr;
    a.Hdense = Hdense;
    a.nk = nk;
    a.nb = nb;
    a.part = part;
    a.err = wait_error_word();
    if (!a.err) return CPPHF_ERR_CUDA;
    if (nb2 <= kTileElems) {
        // whole k-blocks per stage: 1024 elements (3 arrays) or 512 (4 arrays with refP)
        const AsmCfg cfg = kAsmCfg;
        const int elems = refP ? cfg.elems / 2 : cfg.elems;
        const int KT = std::max(1, elems / nb2);
        const int64_t ntiles = (nk + KT - 1) / KT;
        const int narr = refP ? 4 : 3;
        const size_t smem = sizeof(double2) * (size_t)KT * nb2 * narr * cfg.nst + 128;
        static std::once_flag once_b;
        std::call_once(once_b, [] {
            raise_smem(k_assemble_bulk<false, 0>);
            raise_smem(k_assemble_bulk<true, 0>);
            raise_smem(k_assemble_bulk<false, 8>);
            raise_smem(k_assemble_bulk<true, 8>);
        });
        int per = 0;
        if (refP)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_assemble_bulk<true, 0>, kAsmThreads, smem);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_assemble_bulk<false, 0>, kAsmThreads, smem);
        (void)cudaGetLastError();
        per = std::max(1, per);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, std::min<int64_t>(kMaxPartials, (int64_t)per * num_sms())));
        unsigned* counter = reinterpret_cast<unsigned*>(W + L.off_counter);
        if (energy) CPPHF_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
        if (refP && nb == 8)
            k_assemble_bulk<true, 8><<<grid, kAsmThreads, smem, st>>>(a, KT, ntiles, counter, energy, cfg.nst);
        else if (refP)
            k_assemble_bulk<true, 0><<<grid, kAsmThreads, smem, st>>>(a, KT, ntiles, counter, energy, cfg.nst);
        else if (nb == 8)
            k_assemble_bulk<false, 8><<<grid, kAsmThreads, smem, st>>>(a, KT, ntiles, counter, energy, cfg.nst);
        else
            k_assemble_bulk<false, 0><<<grid, kAsmThreads, smem, st>>>(a, KT, ntiles, counter, energy, cfg.nst);
        CPPHF_LAUNCH_CHECK("assemble (bulk pipelined)");
        return CPPHF_OK;
    }
    {
        k_assemble<<<L.Gasm, kAsmThreads, 0, st>>>(a);
        CPPHF_LAUNCH_CHECK("assemble");
    }
    if (energy) {
        k_sum_partials<<<1, 32, 0, st>>>(part, L.Gasm, energy);
        CPPHF_LAUNCH_CHECK("energy sum");
    }
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

size_t cpphf_build_fock_workspace_bytes(const cpphf_kernel* K) {
    return K ? cpphf::build_fock_workspace_bytes(K) : 0;
}

int cpphf_build_fock(const cpphf_kernel* K, const void* P, void* Sigma, void* F, double* hartree_diag,
                     double* energy, void* H_dense, void* workspace, size_t workspace_bytes,
                     void* stream) {
    return cpphf::build_fock(K, static_cast<const double2*>(P), static_cast<double2*>(Sigma),
                             static_cast<double2*>(F), hartree_diag, energy,
                             static_cast<double2*>(H_dense), workspace, workspace_bytes,
                             static_cast<cudaStream_t>(stream));
}

}  // extern "C"
