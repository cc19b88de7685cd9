// Superlattice (moire plane-wave) Fock terms (cpp_hf superlattice.hpp:50-246,
// fock.hpp:66-175).
//
// Streamed exchange: for the plane-wave basis |k + G, alpha>, the Fock
// self-energy decouples into independent Delta-G = G_a - G_b channels, each a
// 2-D convolution in absolute momentum p = k - G on an extended grid of
// (N_ext_x, N_ext_y) points (zero padded so the convolution is aperiodic).
// On the host, the channels to compute are listed (with hermitian_rho a channel
// whose reversed pairs form another channel is computed once and fills both)
// and packed into batches: with a scalar Coulomb table, kq^2 channels of
// dim_orb^2 orbital pairs share one exchange call as a (kq dim_orb)^2 "orbital"
// field, so the mesh exchange kernels (FFT passes through TMA pipelines) run
// unchanged; with an orbital-resolved table each channel is its own call.
// Per batch: zero the extended field, scatter the rho blocks at their tile
// offsets, exchange, gather the blocks (and the conjugate transposes).
//
// Superlattice Hartree: a k-independent nb x nb term from the mean density
// rho_bar, summed over the (G_a, G_b) pairs of each Delta-G channel
// (fock.hpp:66-175), added to the contact matrix that the Fock assembly adds to
// every k-point.
#include "common.cuh"
#include "exchange.cuh"
#include "superlattice.cuh"

#include <algorithm>
#include <map>
#include <string>
#include <vector>

namespace cpphf {

namespace {

struct SlEntry {
    int slot, i, j, partner;
};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct SlPlan {
    int nbf, kq, dv, C;
    std::vector<SlEntry> ent;
    std::vector<int> batch_start;  // entry ranges per batch
};

// rho (x, y, i, a, j, b) -> extended field (ox + x, oy + y, channel of (slot, a, b))
__global__ void k_sl_scatter(const double2* __restrict__ rho, double2* __restrict__ buf,
                             const SlEntry* __restrict__ ent, int n_ent, const int* __restrict__ goff, int nkx,
                             int nky, int nG, int orb, int NY, int C, int nbf, int kq) {
    const int64_t blk = (int64_t)nkx * nky * orb * orb;
    const int64_t total = (int64_t)n_ent * blk;
    const int64_t D = (int64_t)nG * orb;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)(t / blk);
        int64_t r = t - (int64_t)e * blk;
        const int b = (int)(r % orb);
        r /= orb;
        const int a = (int)(r % orb);
        r /= orb;
        const int y = (int)(r % nky);
        const int x = (int)(r / nky);
        const SlEntry en = ent[e];
        const int ox = nkx * goff[2 * en.i], oy = nky * goff[2 * en.i + 1];
        const double2 v = rho[(((int64_t)x * nky + y) * D + (int64_t)en.i * orb + a) * D + (int64_t)en.j * orb + b];
        const int c = ((en.slot / kq) * orb + a) * nbf + (en.slot % kq) * orb + b;
        buf[((int64_t)(ox + x) * NY + (oy + y)) * C + c] = v;
    }
}

// extended field -> sigma blocks (and their conjugate transposes for partners)
__global__ void k_sl_gather(const double2* __restrict__ buf, double2* __restrict__ sigma,
                            const SlEntry* __restrict__ ent, int n_ent, const int* __restrict__ goff, int nkx,
                            int nky, int nG, int orb, int NY, int C, int nbf, int kq) {
    const int64_t blk = (int64_t)nkx * nky * orb * orb;
    const int64_t total = (int64_t)n_ent * blk;
    const int64_t D = (int64_t)nG * orb;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)(t / blk);
        int64_t r = t - (int64_t)e * blk;
        const int b = (int)(r % orb);
        r /= orb;
        const int a = (int)(r % orb);
        r /= orb;
        const int y = (int)(r % nky);
        const int x = (int)(r / nky);
        const SlEntry en = ent[e];
        const int ox = nkx * goff[2 * en.i], oy = nky * goff[2 * en.i + 1];
        const int c = ((en.slot / kq) * orb + a) * nbf + (en.slot % kq) * orb + b;
        const double2 v = buf[((int64_t)(ox + x) * NY + (oy + y)) * C + c];
        const int64_t kxy = (int64_t)x * nky + y;
        sigma[(kxy * D + (int64_t)en.i * orb + a) * D + (int64_t)en.j * orb + b] = v;
        if (en.partner) sigma[(kxy * D + (int64_t)en.j * orb + b) * D + (int64_t)en.i * orb + a] = cconj(v);
    }
}

unsigned grid_for_n(int64_t n) {
    const int64_t want = (n + 255) / 256;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms() * 16));
}

// Channel list (superlattice.hpp:50-246 partner rule) packed into exchange batches.
int make_plan(const int64_t* pair_i, const int64_t* pair_j, const int64_t* pair_start, int64_t n_delta, int64_t nG,
              int64_t orb, bool orbital_vr, bool hermitian, SlPlan& pl) {
    std::vector<int64_t> partner((size_t)n_delta, -1);
    if (hermitian) {
        std::map<std::vector<int64_t>, int64_t> key_to_ch;
        std::vector<std::vector<int64_t>> rkeys((size_t)n_delta);
        for (int64_t d = 0; d < n_delta; ++d) {
            std::vector<int64_t> key, rkey;
            for (int64_t p = pair_start[d]; p < pair_start[d + 1]; ++p) {
                key.push_back(pair_i[p] * nG + pair_j[p]);
                rkey.push_back(pair_j[p] * nG + pair_i[p]);
            }
            std::sort(key.begin(), key.end());
            std::sort(rkey.begin(), rkey.end());
            key_to_ch.emplace(key, d);  // first channel with this key wins
            rkeys[(size_t)d] = rkey;
        }
        for (int64_t d = 0; d < n_delta; ++d) {
            auto it = key_to_ch.find(rkeys[(size_t)d]);
            partner[(size_t)d] = it == key_to_ch.end() ? -1 : it->second;
        }
    }
    if (orbital_vr) {
        pl.kq = 1;
        pl.nbf = (int)orb;
        pl.dv = (int)orb;
    } else {
        pl.kq = orb >= 8 ? 1 : (int)(8 / orb);
        pl.nbf = pl.kq * (int)orb;
        pl.dv = 1;
    }
    pl.C = pl.nbf * pl.nbf;
    const int B = pl.kq * pl.kq;
    pl.ent.clear();
    pl.batch_start.assign(1, 0);
    int slot = 0;
    for (int64_t d = 0; d < n_delta; ++d) {
        const int64_t a = pair_start[d], b = pair_start[d + 1];
        if (a == b) continue;
        const int64_t pr = partner[(size_t)d];
        const bool has = pr >= 0 && pr != d;
        if (has && pr < d) continue;
        for (int64_t p = a; p < b; ++p) {
            if (pair_i[p] < 0 || pair_i[p] >= nG || pair_j[p] < 0 || pair_j[p] >= nG)
                return fail(CPPHF_ERR_INVALID, "pair_i / pair_j entries must lie in [0, n_G)");
            pl.ent.push_back(SlEntry{slot, (int)pair_i[p], (int)pair_j[p], has ? 1 : 0});
        }
        if (++slot == B) {
            pl.batch_start.push_back((int)pl.ent.size());
            slot = 0;
        }
    }
    if (slot != 0) pl.batch_start.push_back((int)pl.ent.size());
    return CPPHF_OK;
}

// fock.hpp:66-175: k-independent superlattice Hartree, added into SC (nb x nb).
__global__ void k_sl_hartree(const double2* __restrict__ rho_bar, const int* __restrict__ p2d, int nG, int orb,
                             int n_delta, double deg, const double* __restrict__ HH_GG,
                             const double* __restrict__ HH_orb, double2* __restrict__ SC, int accumulate,
                             double2* __restrict__ scratch /* n_delta * orb */) {
    const int nb = nG * orb;
    // rho_for_delta[d, g] = sum over (a, b) in channel d of rho_bar[a g, b g]
    // (summed over g as well without an orbital table)
    for (int t = threadIdx.x; t < n_delta * orb; t += blockDim.x) scratch[t] = mk(0.0, 0.0);
    __syncthreads();
    if (threadIdx.x == 0) {  // fixed order, like the reference's pair loop
        for (int a = 0; a < nG; ++a)
            for (int b = 0; b < nG; ++b) {
                const int d = p2d[a * nG + b];
                for (int g = 0; g < orb; ++g) {
                    const double2 v = rho_bar[(a * orb + g) * nb + b * orb + g];
                    const int slot = HH_orb ? d * orb + g : d * orb;
                    scratch[slot] = cadd(scratch[slot], v);
                }
            }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nb * nb; c += blockDim.x) {
        const int I = c / nb, J = c - I * nb;
        const int a = I / orb, x = I - a * orb, b = J / orb, y = J - b * orb;
        double2 v = mk(0.0, 0.0);
        if (x == y) {
            const int d = p2d[a * nG + b];
            if (HH_orb) {
                for (int g = 0; g < orb; ++g)
                    v = cadd(v, cscale(scratch[d * orb + g],
                                       deg * HH_orb[((a * nG + b) * orb + x) * orb + g]));
            } else {
                v = cscale(scratch[d * orb], deg * HH_GG[a * nG + b]);
            }
        }
        SC[c] = accumulate ? cadd(SC[c], v) : v;
    }
}

}  // namespace

size_t superlattice_workspace_bytes(int64_t n_pairs, int64_t nG, int64_t orb, int64_t NX, int64_t NY,
                                    int orbital_vr) {
    const int64_t kq = orbital_vr ? 1 : (orb >= 8 ? 1 : 8 / orb);
    const int64_t C = (kq * orb) * (kq * orb);
    return align256(sizeof(SlEntry) * (size_t)std::max<int64_t>(n_pairs, 1)) +
           align256(sizeof(int) * 2 * (size_t)nG) + 2 * align256(sizeof(double2) * (size_t)NX * NY * C);
}

int superlattice_streamed(const double2* rho, const double2* VR, const double2* VRo, const int64_t* g_a_off,
                          const int64_t* pair_i, const int64_t* pair_j, const int64_t* pair_start, int64_t n_delta,
                          int64_t nkx, int64_t nky, int64_t nG, int64_t orb, int64_t NX, int64_t NY, int hermitian,
                          double2* sigma, void* ws, size_t wsb, cudaStream_t st) {
    if (!rho || !VR || !sigma || !g_a_off || !pair_start) return fail(CPPHF_ERR_INVALID, "superlattice: null pointer");
    if (nkx < 1 || nky < 1 || nG < 1 || orb < 1 || n_delta < 0) return fail(CPPHF_ERR_INVALID, "superlattice: bad sizes");
    const int64_t n_pairs = pair_start[n_delta];
    if (n_pairs > 0 && (!pair_i || !pair_j)) return fail(CPPHF_ERR_INVALID, "superlattice: null pair arrays");
    for (int64_t d = 0; d < n_delta; ++d)
        if (pair_start[d + 1] < pair_start[d]) return fail(CPPHF_ERR_INVALID, "pair_start must be non-decreasing");
    for (int64_t i = 0; i < nG; ++i) {
        const int64_t ox = g_a_off[2 * i], oy = g_a_off[2 * i + 1];
        if (ox < 0 || oy < 0 || (ox + 1) * nkx > NX || (oy + 1) * nky > NY)
            return fail(CPPHF_ERR_INVALID, "g_a_off places a tile outside the extended grid");
    }
    const size_t need = superlattice_workspace_bytes(n_pairs, nG, orb, NX, NY, VRo != nullptr);
    if (!ws || wsb < need)
        return fail(CPPHF_ERR_INVALID, "superlattice: workspace too small (" + std::to_string(need) + " bytes needed)");
    SlPlan pl;
    CPPHF_TRY(make_plan(pair_i, pair_j, pair_start, n_delta, nG, orb, VRo != nullptr, hermitian != 0, pl));
    unsigned char* W = static_cast<unsigned char*>(ws);
    SlEntry* d_ent = reinterpret_cast<SlEntry*>(W);
    size_t off = align256(sizeof(SlEntry) * (size_t)std::max<int64_t>(n_pairs, 1));
    int* d_goff = reinterpret_cast<int*>(W + off);
    off += align256(sizeof(int) * 2 * (size_t)nG);
    const size_t fbytes = sizeof(double2) * (size_t)NX * NY * pl.C;
    double2* buf_in = reinterpret_cast<double2*>(W + off);
    double2* buf_out = reinterpret_cast<double2*>(W + off + align256(fbytes));
    std::vector<int> goff32((size_t)(2 * nG));
    for (int64_t i = 0; i < 2 * nG; ++i) goff32[(size_t)i] = (int)g_a_off[i];
    if (!pl.ent.empty())
        CPPHF_CUDA(cudaMemcpyAsync(d_ent, pl.ent.data(), sizeof(SlEntry) * pl.ent.size(), cudaMemcpyHostToDevice, st));
    CPPHF_CUDA(cudaMemcpyAsync(d_goff, goff32.data(), sizeof(int) * goff32.size(), cudaMemcpyHostToDevice, st));
    const int64_t D = nG * orb;
    CPPHF_CUDA(cudaMemsetAsync(sigma, 0, sizeof(double2) * (size_t)nkx * nky * D * D, st));
    const double2* vr = VRo ? VRo : VR;
    for (size_t bi = 0; bi + 1 < pl.batch_start.size(); ++bi) {
        const int e0 = pl.batch_start[bi], e1 = pl.batch_start[bi + 1];
        const int n_ent = e1 - e0;
        const int64_t work = (int64_t)n_ent * nkx * nky * orb * orb;
        CPPHF_CUDA(cudaMemsetAsync(buf_in, 0, fbytes, st));
        k_sl_scatter<<<grid_for_n(work), 256, 0, st>>>(rho, buf_in, d_ent + e0, n_ent, d_goff, (int)nkx, (int)nky,
                                                      (int)nG, (int)orb, (int)NY, pl.C, pl.nbf, pl.kq);
        CPPHF_LAUNCH_CHECK("superlattice scatter");
        CPPHF_TRY(exchange(buf_in, nullptr, vr, buf_out, NX, NY, pl.nbf, pl.dv, 0, 0, 64, nullptr, 0, st));
        k_sl_gather<<<grid_for_n(work), 256, 0, st>>>(buf_out, sigma, d_ent + e0, n_ent, d_goff, (int)nkx, (int)nky,
                                                     (int)nG, (int)orb, (int)NY, pl.C, pl.nbf, pl.kq);
        CPPHF_LAUNCH_CHECK("superlattice gather");
    }
    // the pageable copies above are staged before cudaMemcpyAsync returns, so
    // the host vectors may go out of scope here
    return CPPHF_OK;
}

namespace {
__global__ void k_field_diff(const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ out,
                             int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = csub(a[i], b[i]);
}
}  // namespace

int field_diff(const double2* a, const double2* b, double2* out, int64_t n, cudaStream_t st) {
    k_field_diff<<<grid_for_n(n), 256, 0, st>>>(a, b, out, n);
    CPPHF_LAUNCH_CHECK("field difference");
    return CPPHF_OK;
}

size_t sl_hartree_workspace_bytes(const cpphf_superlattice* sl) {
    return align256(sizeof(int) * (size_t)(sl->n_G * sl->n_G)) +
           align256(sizeof(double2) * (size_t)(std::max<int64_t>(sl->n_delta, 1) * sl->dim_orb));
}

int sl_hartree(const cpphf_superlattice* sl, const double2* rho_bar, double2* SC, int accumulate, void* ws,
               cudaStream_t st) {
    if (!sl->HH_GG && !sl->HH_GG_orbital) return fail(CPPHF_ERR_INVALID, "superlattice Hartree needs HH_GG");
    if (!sl->pair_to_delta) return fail(CPPHF_ERR_INVALID, "superlattice Hartree needs pair_to_delta");
    const int64_t nG = sl->n_G;
    std::vector<int> p2d((size_t)(nG * nG));
    for (int64_t i = 0; i < nG * nG; ++i) {
        const int64_t d = sl->pair_to_delta[i];
        if (d < 0 || d >= sl->n_delta) return fail(CPPHF_ERR_INVALID, "pair_to_delta entries must lie in [0, n_delta)");
        p2d[(size_t)i] = (int)d;
    }
    unsigned char* W = static_cast<unsigned char*>(ws);
    int* d_p2d = reinterpret_cast<int*>(W);
    double2* scratch = reinterpret_cast<double2*>(W + align256(sizeof(int) * (size_t)(nG * nG)));
    CPPHF_CUDA(cudaMemcpyAsync(d_p2d, p2d.data(), sizeof(int) * p2d.size(), cudaMemcpyHostToDevice, st));
    k_sl_hartree<<<1, 256, 0, st>>>(rho_bar, d_p2d, (int)nG, (int)sl->dim_orb, (int)sl->n_delta,
                                     sl->hartree_degeneracy, sl->HH_GG, sl->HH_GG_orbital, SC, accumulate, scratch);
    CPPHF_LAUNCH_CHECK("superlattice Hartree");
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

size_t cpphf_superlattice_workspace_bytes(int64_t n_pairs, int64_t n_G, int64_t dim_orb, int64_t N_ext_x,
                                          int64_t N_ext_y, int orbital_vr) {
    return cpphf::superlattice_workspace_bytes(n_pairs, n_G, dim_orb, N_ext_x, N_ext_y, orbital_vr);
}

int cpphf_superlattice_streamed(const void* rho, const void* V_lag_fft, const void* V_lag_fft_orbital,
                                const int64_t* g_a_off, const int64_t* pair_i, const int64_t* pair_j,
                                const int64_t* pair_start, int64_t n_delta, int64_t nkx, int64_t nky,
                                int64_t n_G, int64_t dim_orb, int64_t N_ext_x, int64_t N_ext_y,
                                int hermitian_rho, void* sigma, void* workspace, size_t workspace_bytes,
                                void* stream) {
    return cpphf::superlattice_streamed(static_cast<const double2*>(rho), static_cast<const double2*>(V_lag_fft),
                                        static_cast<const double2*>(V_lag_fft_orbital), g_a_off, pair_i, pair_j,
                                        pair_start, n_delta, nkx, nky, n_G, dim_orb, N_ext_x, N_ext_y, hermitian_rho,
                                        static_cast<double2*>(sigma), workspace, workspace_bytes,
                                        static_cast<cudaStream_t>(stream));
}

}  // extern "C"
