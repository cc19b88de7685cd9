// Derivative kernels for the differentiable Fock-build API: the pieces that
// torch.autograd.Function wrappers of build_fock, hf_energy, free_energy and
// density_from_fock call in their forward and backward passes.
//
// The reference computes these quantities without derivatives
// (cpp_hf fock.py:16-124, fock.hpp:324-407, solver_scf.hpp:96-154); the
// backward formulas here follow from those definitions:
//   E = sum_k w_k Re[ Tr(h P) + 1/2 Tr((Sigma + H)(P - refP)) ]
//   S = -sum_k w_k sum_i [p ln p + (1 - p) ln(1 - p)],  p clipped to [1e-14, 1 - 1e-14]
//   P = V f((mu - eps)/T) V^H with mu fixed by sum_k w_k sum_i f = n_e.
// Gradients use torch's convention for complex tensors: for a real loss L,
// grad z = dL/dRe z + i dL/dIm z.
#include "common.cuh"
#include "dm.cuh"
#include "eigh.cuh"
#include "mu.cuh"
#include "team.cuh"

#include <algorithm>
#include <mutex>
#include <string>

namespace cpphf {

namespace {

constexpr double kPClip = 1.0e-14;  // fock.py:110-113 (occupation_entropy clip)
constexpr int kGradMaxBlocks = 1024;

struct ReduceWs {
    double part[2 * kGradMaxBlocks];
    unsigned counter;
    unsigned pad[63];
};


unsigned red_grid(int64_t n) {
    const int64_t want = (n + 255) / 256;
    const int64_t cap = std::min<int64_t>(kGradMaxBlocks, (int64_t)num_sms() * 4);
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, cap));
}

__device__ __forceinline__ double expit_g(double x) {
    if (x >= 0.0) return 1.0 / (1.0 + exp(-x));
    const double e = exp(x);
    return e / (1.0 + e);
}

// ---------------------------------------------------------------------------
// build_fock backward prep: hF = herm(gF); gS = gSigma + hF; gh = hF
// ---------------------------------------------------------------------------
__global__ void k_fock_bwd_prep(const double2* __restrict__ gSig, const double2* __restrict__ gF, double2* gS,
                                double2* gh, int64_t nk, int nb) {
    const int npair = nb * (nb + 1) / 2;
    const int64_t total = nk * npair;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t / npair;
        int r = (int)(t - k * npair), i = 0;
        while (r >= nb - i) {
            r -= nb - i;
            ++i;
        }
        const int j = i + r;
        const size_t ij = (size_t)k * nb * nb + (size_t)i * nb + j, ji = (size_t)k * nb * nb + (size_t)j * nb + i;
        double2 hij = mk(0.0, 0.0);
        if (gF) {
            const double2 a = gF[ij], b = gF[ji];
            hij = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        }
        const double2 hji = cconj(hij);
        if (gS) {
            gS[ij] = gSig ? cadd(gSig[ij], hij) : hij;
            if (ji != ij) gS[ji] = gSig ? cadd(gSig[ji], hji) : hji;
        }
        if (gh) {
            gh[ij] = hij;
            gh[ji] = hji;
        }
    }
}

// ---------------------------------------------------------------------------
// hf_energy forward (fock.hpp:324-383 / fock.py:91-107)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 h_at(const double2* H, int per_k, int64_t k, int nb, int i, int j) {
    return per_k ? H[((size_t)k * nb + i) * nb + j] : H[(size_t)i * nb + j];
}

__global__ void __launch_bounds__(256) k_hf_energy(const double2* __restrict__ h, const double2* __restrict__ Sig,
                                                   const double2* __restrict__ H, int H_per_k,
                                                   const double2* __restrict__ P, const double2* __restrict__ refP,
                                                   const double* __restrict__ w, int64_t nk, int nb, ReduceWs* R,
                                                   double* E) {
    __shared__ double red[32];
    const int64_t nb2 = (int64_t)nb * nb, total = nk * nb2;
    Kahan acc;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / nb2;
        const int r = (int)(e - k * nb2), i = r / nb, j = r - i * nb;
        const size_t ji = (size_t)k * nb2 + (size_t)j * nb + i;
        const double2 pji = P[ji];
        const double2 dji = refP ? csub(pji, refP[ji]) : pji;
        double2 s = Sig ? Sig[e] : mk(0.0, 0.0);
        if (H) s = cadd(s, h_at(H, H_per_k, k, nb, i, j));
        const double2 hv = h[e];
        // Re(h_ij P_ji) + 1/2 Re(s_ij dP_ji)
        const double term = (hv.x * pji.x - hv.y * pji.y) + 0.5 * (s.x * dji.x - s.y * dji.y);
        acc.add(w[k] * term);
    }
    double v[1] = {acc.s};
    double out[1];
    if (reduce_last_block<1>(v, R->part, &R->counter, out, red) && threadIdx.x == 0) *E = out[0];
}

// elementwise gradients of E; gE is a device scalar
__global__ void k_hf_energy_bwd(const double2* __restrict__ h, const double2* __restrict__ Sig,
                                const double2* __restrict__ H, int H_per_k, const double2* __restrict__ P,
                                const double2* __restrict__ refP, const double* __restrict__ w,
                                const double* __restrict__ gE, int64_t nk, int nb, double2* gP, double2* gh,
                                double2* gSig, double2* gHk, double2* grefP) {
    const double ge = *gE;
    const int64_t nb2 = (int64_t)nb * nb, total = nk * nb2;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / nb2;
        const int r = (int)(e - k * nb2), i = r / nb, j = r - i * nb;
        const size_t ji = (size_t)k * nb2 + (size_t)j * nb + i;
        const double c = ge * w[k];
        if (gP || grefP) {
            double2 sji = Sig ? Sig[ji] : mk(0.0, 0.0);
            if (H) sji = cadd(sji, h_at(H, H_per_k, k, nb, j, i));
            if (gP) gP[e] = cscale(cconj(cadd(h[ji], cscale(sji, 0.5))), c);
            if (grefP) grefP[e] = cscale(cconj(sji), -0.5 * c);
        }
        if (gh || gSig || gHk) {
            const double2 pji = P[ji];
            if (gh) gh[e] = cscale(cconj(pji), c);
            const double2 dji = refP ? csub(pji, refP[ji]) : pji;
            const double2 g = cscale(cconj(dji), 0.5 * c);
            if (gSig) gSig[e] = g;
            if (gHk) gHk[e] = g;
        }
    }
}

// shared (k-independent) H: gH_ij = 1/2 gE sum_k w_k conj(dP_k,ji); one block per (i, j)
__global__ void __launch_bounds__(256) k_hf_energy_bwd_shared_h(const double2* __restrict__ P,
                                                                const double2* __restrict__ refP,
                                                                const double* __restrict__ w,
                                                                const double* __restrict__ gE, int64_t nk, int nb,
                                                                double2* gH) {
    __shared__ double red[64];
    const int ij = blockIdx.x, i = ij / nb, j = ij - i * nb;
    const size_t nb2 = (size_t)nb * nb;
    Kahan ar, ai;
    for (int64_t k = threadIdx.x; k < nk; k += blockDim.x) {
        const size_t ji = (size_t)k * nb2 + (size_t)j * nb + i;
        double2 d = P[ji];
        if (refP) d = csub(d, refP[ji]);
        ar.add(w[k] * d.x);
        ai.add(-w[k] * d.y);
    }
    double v[2] = {ar.s, ai.s};
    block_sum<2>(v, red);
    if (threadIdx.x == 0) gH[ij] = mk(0.5 * (*gE) * v[0], 0.5 * (*gE) * v[1]);
}

// ---------------------------------------------------------------------------
// occupation entropy (fock.hpp:385-407 / fock.py:110-115)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_entropy(const double* __restrict__ p, const double* __restrict__ wn,
                                                 int64_t nk, int nb, ReduceWs* R, double* S) {
    __shared__ double red[32];
    const int64_t total = nk * nb;
    Kahan acc;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const double ps = fmin(fmax(p[e], kPClip), 1.0 - kPClip);
        acc.add(wn[e / nb] * (ps * log(ps) + (1.0 - ps) * log1p(-ps)));
    }
    double v[1] = {acc.s};
    double out[1];
    if (reduce_last_block<1>(v, R->part, &R->counter, out, red) && threadIdx.x == 0) *S = -out[0];
}

// dS/dp = -w (ln p - ln(1 - p)) inside the clip window, 0 outside
__global__ void k_entropy_bwd(const double* __restrict__ p, const double* __restrict__ wn,
                              const double* __restrict__ gS, int64_t nk, int nb, double* __restrict__ gp) {
    const double g = *gS;
    const int64_t total = nk * nb;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const double x = p[e];
        double d = 0.0;
        if (x > kPClip && x < 1.0 - kPClip) d = -wn[e / nb] * (log(x) - log1p(-x));
        gp[e] = g * d;
    }
}

// ---------------------------------------------------------------------------
// density_from_fock backward.  With f_i = expit((mu - eps_i)/T) and mu fixed by
// the electron count, a Hermitian perturbation dF gives, in the eigenbasis
// (dF~ = V^H dF V):
//   dP~_ij = D_ij dF~_ij,   D_ij = (f_i - f_j)/(eps_i - eps_j),  D_ii = f'_i
//   minus the mu shift on the diagonal: dP~_ii -= f'_i dmu,
//   dmu = sum_k w_k sum_i f'_i dF~_ii / sum_k w_k sum_i f'_i.
// The map is self-adjoint except for the mu term, whose adjoint puts
// -w_k f'_i A / Z on the diagonal with A = sum_{k,i} Re(G~_ii) f'_i and
// Z = sum_k w_k sum_i f'_i.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double fd_divided(double ei, double ej, double mu, double T) {
    const double s = (ei - ej) / (2.0 * T);
    if (fabs(s) > 1.0e-3) {
        const double fi = expit_g((mu - ei) / T), fj = expit_g((mu - ej) / T);
        return (fi - fj) / (ei - ej);
    }
    // f(x) = (1 - tanh(a))/2 with a = (e - mu)/(2T):
    // f_i - f_j = -sinh(a_i - a_j) / (2 cosh a_i cosh a_j), cosh a_i cosh a_j = (cosh(a_i + a_j) + cosh s)/2
    const double ssum = (ei + ej - 2.0 * mu) / (2.0 * T);
    if (fabs(ssum) > 1400.0) return 0.0;
    const double sinhc = 1.0 + s * s / 6.0 * (1.0 + s * s / 20.0);  // sinh(s)/s, |s| <= 1e-3
    return -sinhc / (2.0 * T * (cosh(ssum) + cosh(s)));
}

template <bool WARP>
__global__ void k_dff_bwd_rotate(const double2* __restrict__ V, const double* __restrict__ eps,
                                 const double* __restrict__ mu, double T, const double* __restrict__ w,
                                 const double2* __restrict__ G, double2* __restrict__ Gt, int64_t nk, int nb,
                                 ReduceWs* R, double* AZ) {
    extern __shared__ __align__(16) unsigned char raw[];
    __shared__ double red[64];
    Team<WARP> t;
    const int ld = nb + 1;
    double2* Vs = team_mats<WARP>(raw, nb, 3, 0, t.team);
    double2* Gs = Vs + team_mat_elems(nb);
    double2* Ts = Gs + team_mat_elems(nb);
    const double m = *mu;
    double v[2] = {0.0, 0.0};
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Vs, V + (size_t)k * nb * nb, nb, t);
        const double2* Gk = G + (size_t)k * nb * nb;
        for (int e = t.tid; e < nb * nb; e += t.nt) {  // herm(G)
            const int i = e / nb, j = e - i * nb;
            const double2 a = Gk[e], b = Gk[(size_t)j * nb + i];
            Gs[i * ld + j] = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        }
        t.sync();
        tmm<false, false, WARP>(Ts, Gs, Vs, nb, t);  // herm(G) V
        t.sync();
        tmm<true, false, WARP>(Gs, Vs, Ts, nb, t);   // V^H herm(G) V
        t.sync();
        tstore<WARP>(Gt + (size_t)k * nb * nb, Gs, nb, t);
        for (int i = t.tid; i < nb; i += t.nt) {
            const double f = expit_g((m - eps[(size_t)k * nb + i]) / T);
            const double fp = -f * (1.0 - f) / T;
            v[0] += Gs[i * ld + i].x * fp;
            v[1] += w[k] * fp;
        }
        t.sync();
    }
    double out[2];
    if (reduce_last_block<2>(v, R->part, &R->counter, out, red) && threadIdx.x == 0) {
        AZ[0] = out[0];
        AZ[1] = out[1];
    }
}

template <bool WARP>
__global__ void k_dff_bwd_apply(const double2* __restrict__ V, const double* __restrict__ eps,
                                const double* __restrict__ mu, double T, const double* __restrict__ w,
                                const double* __restrict__ AZ, double2* gF, int64_t nk, int nb) {
    extern __shared__ __align__(16) unsigned char raw[];
    Team<WARP> t;
    const int ld = nb + 1;
    double2* Vs = team_mats<WARP>(raw, nb, 3, nb, t.team);
    double2* Ms = Vs + team_mat_elems(nb);
    double2* Ts = Ms + team_mat_elems(nb);
    double* es = reinterpret_cast<double*>(Ts + team_mat_elems(nb));
    const double m = *mu;
    const double Z = AZ[1];
    const double ratio = (fabs(Z) > 1.0e-300) ? AZ[0] / Z : 0.0;
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Vs, V + (size_t)k * nb * nb, nb, t);
        tload<WARP>(Ms, gF + (size_t)k * nb * nb, nb, t);
        for (int i = t.tid; i < nb; i += t.nt) es[i] = eps[(size_t)k * nb + i];
        t.sync();
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            double d = fd_divided(es[i], es[j], m, T);
            double2 x = cscale(Ms[i * ld + j], d);
            if (i == j) {
                const double f = expit_g((m - es[i]) / T);
                x.x -= w[k] * (-f * (1.0 - f) / T) * ratio;
            }
            Ms[i * ld + j] = x;
        }
        t.sync();
        tmm<false, true, WARP>(Ts, Ms, Vs, nb, t);   // M V^H
        t.sync();
        tmm<false, false, WARP>(Ms, Vs, Ts, nb, t);  // V M V^H
        t.sync();
        tstore<WARP>(gF + (size_t)k * nb * nb, Ms, nb, t);
        t.sync();
    }
}

void init_grad_attrs() {
    static std::once_flag once;
    std::call_once(once, [] {
        raise_smem(k_dff_bwd_rotate<true>);
        raise_smem(k_dff_bwd_rotate<false>);
        raise_smem(k_dff_bwd_apply<true>);
        raise_smem(k_dff_bwd_apply<false>);
    });
}

int check_sizes(int64_t nk, int64_t nb) {
    if (nk < 1 || nb < 1) return fail(CPPHF_ERR_INVALID, "empty mesh or nb");
    return CPPHF_OK;
}

}  // namespace

size_t reduce_workspace_bytes() { return sizeof(ReduceWs); }

int fock_backward_prep(const double2* gSig, const double2* gF, double2* gS, double2* gh, int64_t nk, int64_t nb,
                       cudaStream_t st) {
    CPPHF_TRY(check_sizes(nk, nb));
    const int64_t tot = nk * nb * (nb + 1) / 2;
    k_fock_bwd_prep<<<red_grid(tot) * 4, 256, 0, st>>>(gSig, gF, gS, gh, nk, (int)nb);
    CPPHF_LAUNCH_CHECK("fock backward prep");
    return CPPHF_OK;
}

int hf_energy(const double2* h, const double2* Sig, const double2* H, int H_per_k, const double2* P,
              const double2* refP, const double* w, int64_t nk, int64_t nb, double* E, void* ws, size_t wsb,
              cudaStream_t st) {
    CPPHF_TRY(check_sizes(nk, nb));
    if (!h || !P || !w || !E) return fail(CPPHF_ERR_INVALID, "hf_energy: null pointer");
    if (!ws || wsb < sizeof(ReduceWs)) return fail(CPPHF_ERR_INVALID, "hf_energy: workspace too small");
    ReduceWs* R = static_cast<ReduceWs*>(ws);
    CPPHF_CUDA(cudaMemsetAsync(&R->counter, 0, sizeof(unsigned), st));
    k_hf_energy<<<red_grid(nk * nb * nb), 256, 0, st>>>(h, Sig, H, H_per_k, P, refP, w, nk, (int)nb, R, E);
    CPPHF_LAUNCH_CHECK("hf_energy");
    return CPPHF_OK;
}

int hf_energy_backward(const double2* h, const double2* Sig, const double2* H, int H_per_k, const double2* P,
                       const double2* refP, const double* w, const double* gE, int64_t nk, int64_t nb, double2* gP,
                       double2* gh, double2* gSig, double2* gH, double2* grefP, cudaStream_t st) {
    CPPHF_TRY(check_sizes(nk, nb));
    if (!h || !P || !w || !gE) return fail(CPPHF_ERR_INVALID, "hf_energy_backward: null pointer");
    k_hf_energy_bwd<<<red_grid(nk * nb * nb) * 4, 256, 0, st>>>(h, Sig, H, H_per_k, P, refP, w, gE, nk, (int)nb, gP,
                                                               gh, gSig, H_per_k ? gH : nullptr, grefP);
    CPPHF_LAUNCH_CHECK("hf_energy backward");
    if (gH && !H_per_k) {
        k_hf_energy_bwd_shared_h<<<(unsigned)(nb * nb), 256, 0, st>>>(P, refP, w, gE, nk, (int)nb, gH);
        CPPHF_LAUNCH_CHECK("hf_energy backward (shared H)");
    }
    return CPPHF_OK;
}

int occupation_entropy(const double* p, const double* wn, int64_t nk, int64_t nb, double* S, void* ws, size_t wsb,
                       cudaStream_t st) {
    CPPHF_TRY(check_sizes(nk, nb));
    if (!p || !wn || !S) return fail(CPPHF_ERR_INVALID, "occupation_entropy: null pointer");
    if (!ws || wsb < sizeof(ReduceWs)) return fail(CPPHF_ERR_INVALID, "occupation_entropy: workspace too small");
    ReduceWs* R = static_cast<ReduceWs*>(ws);
    CPPHF_CUDA(cudaMemsetAsync(&R->counter, 0, sizeof(unsigned), st));
    k_entropy<<<red_grid(nk * nb), 256, 0, st>>>(p, wn, nk, (int)nb, R, S);
    CPPHF_LAUNCH_CHECK("occupation_entropy");
    return CPPHF_OK;
}

int occupation_entropy_backward(const double* p, const double* wn, const double* gS, int64_t nk, int64_t nb,
                                double* gp, cudaStream_t st) {
    CPPHF_TRY(check_sizes(nk, nb));
    if (!p || !wn || !gS || !gp) return fail(CPPHF_ERR_INVALID, "occupation_entropy_backward: null pointer");
    k_entropy_bwd<<<red_grid(nk * nb) * 4, 256, 0, st>>>(p, wn, gS, nk, (int)nb, gp);
    CPPHF_LAUNCH_CHECK("occupation_entropy backward");
    return CPPHF_OK;
}

size_t density_from_fock_backward_workspace_bytes() { return sizeof(ReduceWs) + 256; }

int density_from_fock_backward(const double2* V, const double* eps, const double* mu, double T, const double* w,
                               const double2* G, double2* gF, int64_t nk, int64_t nb, void* ws, size_t wsb,
                               cudaStream_t st) {
    CPPHF_TRY(check_sizes(nk, nb));
    CPPHF_TRY(dm_check_nb(nb));
    if (!V || !eps || !mu || !w || !G || !gF) return fail(CPPHF_ERR_INVALID, "density_from_fock_backward: null pointer");
    if (!(T > 0.0)) return fail(CPPHF_ERR_INVALID, "density_from_fock_backward: T must be positive");
    if (!ws || wsb < density_from_fock_backward_workspace_bytes())
        return fail(CPPHF_ERR_INVALID, "density_from_fock_backward: workspace too small");
    init_grad_attrs();
    ReduceWs* R = static_cast<ReduceWs*>(ws);
    double* AZ = reinterpret_cast<double*>(static_cast<unsigned char*>(ws) + sizeof(ReduceWs));
    CPPHF_CUDA(cudaMemsetAsync(&R->counter, 0, sizeof(unsigned), st));
    TeamLaunch L = team_launch(nk, (int)nb);
    L.grid = std::min<unsigned>(L.grid, kGradMaxBlocks);
    const int n = (int)nb;
    {
        const int nb = n;  // for TEAM_DISPATCH's shared-memory size
        TEAM_DISPATCH(L, k_dff_bwd_rotate, 3, 0, V, eps, mu, T, w, G, gF, nk, n, R, AZ);
        TEAM_DISPATCH(L, k_dff_bwd_apply, 3, nb, V, eps, mu, T, w, AZ, gF, nk, n);
    }
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

size_t cpphf_reduce_workspace_bytes(void) { return cpphf::reduce_workspace_bytes(); }

int cpphf_fock_backward_prep(const void* gSigma, const void* gF, void* gS, void* gh, int64_t nk, int64_t nb,
                             void* stream) {
    return cpphf::fock_backward_prep(static_cast<const double2*>(gSigma), static_cast<const double2*>(gF),
                                     static_cast<double2*>(gS), static_cast<double2*>(gh), nk, nb,
                                     static_cast<cudaStream_t>(stream));
}

int cpphf_hf_energy(const void* h, const void* Sigma, const void* H, int H_per_k, const void* P, const void* refP,
                    const double* w, int64_t nk, int64_t nb, double* E, void* workspace, size_t workspace_bytes,
                    void* stream) {
    return cpphf::hf_energy(static_cast<const double2*>(h), static_cast<const double2*>(Sigma),
                            static_cast<const double2*>(H), H_per_k, static_cast<const double2*>(P),
                            static_cast<const double2*>(refP), w, nk, nb, E, workspace, workspace_bytes,
                            static_cast<cudaStream_t>(stream));
}

int cpphf_hf_energy_backward(const void* h, const void* Sigma, const void* H, int H_per_k, const void* P,
                             const void* refP, const double* w, const double* gE, int64_t nk, int64_t nb, void* gP,
                             void* gh, void* gSigma, void* gH, void* grefP, void* stream) {
    return cpphf::hf_energy_backward(static_cast<const double2*>(h), static_cast<const double2*>(Sigma),
                                     static_cast<const double2*>(H), H_per_k, static_cast<const double2*>(P),
                                     static_cast<const double2*>(refP), w, gE, nk, nb, static_cast<double2*>(gP),
                                     static_cast<double2*>(gh), static_cast<double2*>(gSigma),
                                     static_cast<double2*>(gH), static_cast<double2*>(grefP),
                                     static_cast<cudaStream_t>(stream));
}

int cpphf_occupation_entropy(const double* p, const double* w_norm, int64_t nk, int64_t nb, double* S,
                             void* workspace, size_t workspace_bytes, void* stream) {
    return cpphf::occupation_entropy(p, w_norm, nk, nb, S, workspace, workspace_bytes,
                                     static_cast<cudaStream_t>(stream));
}

int cpphf_occupation_entropy_backward(const double* p, const double* w_norm, const double* gS, int64_t nk, int64_t nb,
                                      double* gp, void* stream) {
    return cpphf::occupation_entropy_backward(p, w_norm, gS, nk, nb, gp, static_cast<cudaStream_t>(stream));
}

size_t cpphf_density_from_fock_backward_workspace_bytes(void) {
    return cpphf::density_from_fock_backward_workspace_bytes();
}

int cpphf_density_from_fock_backward(const void* V, const double* eps, const double* mu, double T, const double* w,
                                     const void* G, void* gF, int64_t nk, int64_t nb, void* workspace,
                                     size_t workspace_bytes, void* stream) {
    return cpphf::density_from_fock_backward(static_cast<const double2*>(V), eps, mu, T, w,
                                             static_cast<const double2*>(G), static_cast<double2*>(gF), nk, nb,
                                             workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
