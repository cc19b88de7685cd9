// Solver loops on device-resident state: direct minimisation
// (cpp_hf solver_dm.hpp:392-653, optimizer "cg") and SCF with linear mixing
// (solver_scf.hpp:96-444).  The host replays the reference's control flow
// (fixed iteration rules, plateau window, strict acceptance); every array
// operation is a kernel on `stream`, and each iteration reads back only the
// few scalars its convergence test needs.
#include "common.cuh"
#include "dm.cuh"
#include "dm_small.cuh"
#include "eigh.cuh"
#include "fock.cuh"
#include "mu.cuh"
#include "team.cuh"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

namespace cpphf {

namespace {

constexpr double TINY_REAL = 1.0e-30;

__global__ void k_scale_weights(const double* __restrict__ w, double inv, double* __restrict__ out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = w[i] / inv;
}

// in-place hermitisation of (nk, nb, nb); optionally copying from src first
__global__ void k_hermitize(const double2* src, double2* dst, int64_t nk, int nb) {
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
        const double2 a = src[ij], b = src[ji];
        const double2 h = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        dst[ij] = h;
        dst[ji] = cconj(h);
    }
}

__global__ void k_set_scalar(double* p, double v) { *p = v; }

// level-shifted SCF occupations (solver_scf.hpp:127-141):
// shifted = eps + ls (1 - f(eps - mu_raw)); output occ = f(shifted - mu) later.
__device__ __forceinline__ double expit_d(double x) {
    if (x >= 0.0) return 1.0 / (1.0 + exp(-x));
    const double e = exp(x);
    return e / (1.0 + e);
}

__global__ void k_level_shift(const double* __restrict__ eps, const double* __restrict__ mu_raw, double T, double ls,
                              double* __restrict__ shifted, int64_t n) {
    const double m = *mu_raw;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double occ = expit_d(-(eps[i] - m) / (T + 1.0e-12));
        shifted[i] = eps[i] + ls * (1.0 - occ);
    }
}

__global__ void k_fermi(const double* __restrict__ e, const double* __restrict__ mu, double T, double* __restrict__ occ,
                        int64_t n) {
    const double m = *mu;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        occ[i] = expit_d(-(e[i] - m) / (T + 1.0e-12));
}

// SCF residuals: delta = P_new - D, comm = F D - D F; weighted squared norms.
// One team per k (solver_scf.hpp:224-242, 64-75).
template <bool WARP>
__global__ void k_scf_residuals(const double2* __restrict__ F, const double2* __restrict__ D,
                                const double2* __restrict__ Pn, const double* __restrict__ w, int64_t nk, int nb,
                                DmScalars* S) {
    extern __shared__ __align__(16) unsigned char raw[];
    __shared__ double red[64];
    Team<WARP> t;
    const int ld = nb + 1;
    const size_t per = (sizeof(double2) * team_mat_elems(nb) * 2 + 15) & ~(size_t)15;
    double2* Fs = reinterpret_cast<double2*>(raw + per * t.team);
    double2* Ds = Fs + team_mat_elems(nb);
    double v[2] = {0.0, 0.0};
    for (int64_t k = (int64_t)blockIdx.x * t.nteams + t.team; k < nk; k += (int64_t)gridDim.x * t.nteams) {
        tload<WARP>(Fs, F + (size_t)k * nb * nb, nb, t);
        tload<WARP>(Ds, D + (size_t)k * nb * nb, nb, t);
        t.sync();
        const double wk = w[k];
        double sd = 0.0, sc = 0.0;
        for (int e = t.tid; e < nb * nb; e += t.nt) {
            const int i = e / nb, j = e - i * nb;
            const double2 d = csub(Pn[(size_t)k * nb * nb + e], Ds[i * ld + j]);
            sd += d.x * d.x + d.y * d.y;
            double2 fp = mk(0.0, 0.0), pf = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) {
                cfma(fp, Fs[i * ld + l], Ds[l * ld + j]);
                cfma(pf, Ds[i * ld + l], Fs[l * ld + j]);
            }
            const double2 c = csub(fp, pf);
            sc += c.x * c.x + c.y * c.y;
        }
        v[0] += wk * sd;
        v[1] += wk * sc;
        t.sync();
    }
    double out[2];
    if (reduce_last_block<2>(v, S->part, &S->counter, out, red) && threadIdx.x == 0) {
        S->grad_norm = out[0];  // density residual^2 * weight_sum
        S->lam_pc = out[1];     // commutator residual^2 * weight_sum
    }
}

// density <- herm(density + mixing (P_new - density))  (solver_scf.hpp:395-401)
__global__ void k_scf_mix(double2* D, const double2* __restrict__ Pn, double mixing, int64_t nk, int nb) {
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
        const double2 dij = D[ij], dji = D[ji];
        const double2 a = cadd(dij, cscale(csub(Pn[ij], dij), mixing));
        const double2 b = cadd(dji, cscale(csub(Pn[ji], dji), mixing));
        const double2 h = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        D[ij] = h;
        D[ji] = cconj(h);
    }
}

unsigned grid_for(int64_t n, int threads) {
    const int64_t want = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms() * 8));
}

int hermitize(const double2* src, double2* dst, int64_t nk, int nb, cudaStream_t st) {
    const int64_t tot = nk * (int64_t)nb * (nb + 1) / 2;
    k_hermitize<<<grid_for(tot, 256), 256, 0, st>>>(src, dst, nk, nb);
    CPPHF_LAUNCH_CHECK("hermitize");
    return CPPHF_OK;
}

int call_project(cpphf_project_fn fn, void* user, double2* M, const cpphf_kernel* K, cudaStream_t st) {
    if (!fn) return CPPHF_OK;
    const int rc = fn(user, M, K->nk1, K->nk2, K->nb, st);
    if (rc != 0) return fail(CPPHF_ERR_INVALID, std::string("project_fn failed: ") + cpphf_last_error());
    return CPPHF_OK;
}

// Workspace carve-up shared by both solvers.
struct SolverWs {
    size_t total = 0;
    size_t take(size_t bytes) {
        const size_t at = total;
        total += (bytes + 255) & ~(size_t)255;
        return at;
    }
};

// Fock workspace large enough for the complex64 and the complex128 exchange, so
// a switched-precision solve can build in either form from one workspace.
size_t fock_bytes_any_precision(const cpphf_kernel* K) {
    cpphf_kernel K32 = *K;
    K32.exchange_precision = 32;
    return std::max(build_fock_workspace_bytes(K), build_fock_workspace_bytes(&K32));
}

// Exchange precision of a switched solve: complex64 first, complex128 after.
int check_mixed(const cpphf_kernel* K, double sw) {
    if (!(sw >= 0.0)) return fail(CPPHF_ERR_INVALID, "mixed-precision switch threshold must be >= 0");
    if (sw > 0.0 && K->exchange_precision != 64)
        return fail(CPPHF_ERR_INVALID, "a switched-precision solve needs exchange_precision 64 in the kernel");
    return CPPHF_OK;
}

struct DmLayout {
    size_t Q, P, Sig, F, G[2], dQ[2], Vd, p, eps, g[2], dp[2], lam, ew, wn, S, fock_ws, mu_ws, total;
    size_t fock_bytes, mu_bytes;
};

DmLayout dm_layout(const cpphf_kernel* K) {
    const size_t nk = (size_t)K->nk1 * K->nk2, nb = (size_t)K->nb;
    const size_t fld = sizeof(double2) * nk * nb * nb, vec = sizeof(double) * nk * nb;
    SolverWs W;
    DmLayout L;
    L.Q = W.take(fld);
    L.P = W.take(fld);
    L.Sig = W.take(fld);
    L.F = W.take(fld);
    L.G[0] = W.take(fld);
    L.G[1] = W.take(fld);
    L.dQ[0] = W.take(fld);
    L.dQ[1] = W.take(fld);
    L.Vd = W.take(fld);
    L.p = W.take(vec);
    L.eps = W.take(vec);
    L.g[0] = W.take(vec);
    L.g[1] = W.take(vec);
    L.dp[0] = W.take(vec);
    L.dp[1] = W.take(vec);
    L.lam = W.take(vec);
    L.ew = W.take(vec);
    L.wn = W.take(sizeof(double) * nk);
    L.S = W.take(sizeof(DmScalars));
    L.fock_bytes = fock_bytes_any_precision(K);
    L.fock_ws = W.take(L.fock_bytes);
    L.mu_bytes = mu_workspace_bytes((int64_t)nk, (int64_t)nb);
    L.mu_ws = W.take(L.mu_bytes);
    L.total = W.total;
    return L;
}

int check_block_sizes(const int64_t* sizes, int64_t n, int64_t nb) {
    if (n <= 0) return CPPHF_OK;
    int64_t tot = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (sizes[i] == 0) return fail(CPPHF_ERR_INVALID, "block_sizes entries must be positive.");
        tot += sizes[i];
    }
    if (tot != nb) return fail(CPPHF_ERR_INVALID, "block_sizes must sum to nb.");
    return CPPHF_OK;
}

// The legacy default stream cannot be captured: a solve called on it runs on
// its own non-blocking stream, ordered after the caller's stream on entry and
// before it on exit.  A solve on any other stream runs (and is captured) on
// that stream directly.  `capturable` is false when the private stream could
// not be created; the solve then runs on the caller's stream without graphs.
struct SolveStream {
    cudaStream_t user = nullptr, s = nullptr;
    cudaEvent_t ev = nullptr;
    bool capturable = true;
    explicit SolveStream(cudaStream_t u) : user(u) {
        if (u != nullptr && u != cudaStreamLegacy) return;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventRecord(ev, user) != cudaSuccess || cudaStreamWaitEvent(s, ev, 0) != cudaSuccess) {
            (void)cudaGetLastError();
            if (s) cudaStreamDestroy(s);
            s = nullptr;
            capturable = false;
        }
    }
    ~SolveStream() {
        if (s) {
            cudaEventRecord(ev, s);
            cudaStreamWaitEvent(user, ev, 0);
            cudaStreamDestroy(s);
        }
        if (ev) cudaEventDestroy(ev);
    }
    cudaStream_t stream() const { return s ? s : user; }
};

// One DM iteration as an instantiated graph, per (buffer parity, precision).
struct IterGraphs {
    cudaGraphExec_t exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    bool failed[2][2] = {{false, false}, {false, false}};
    ~IterGraphs() {
        for (auto& row : exec)
            for (auto& e : row)
                if (e) cudaGraphExecDestroy(e);
    }
};

// CPPHF_SOLVE_GRAPHS=0 launches every kernel of every iteration (for A/B timing).
bool solve_graphs_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("CPPHF_SOLVE_GRAPHS");
        return !(e && e[0] == '0');
    }();
    return on;
}

}  // namespace

size_t solve_dm_workspace_bytes(const cpphf_kernel* K) { return dm_layout(K).total; }

int solve_dm(const cpphf_kernel* K, const cpphf_dm_config* cfg, const double2* P0, double n_e,
             cpphf_project_fn project, void* puser, double2* Q_out, double* p_out, double2* D_out, double2* F_out,
             double* hist_E, double* hist_G, cpphf_dm_result* res, void* ws, size_t wsb, cudaStream_t st) {
    CPPHF_TRY(validate_kernel(K));
    if (!cfg || !P0 || !res) return fail(CPPHF_ERR_INVALID, "solve_dm: null argument");
    if (cfg->optimizer != 0)
        return fail(CPPHF_ERR_UNSUPPORTED, "optimizer='newton' (trust-region Newton) is not built into this library");
    CPPHF_TRY(check_block_sizes(cfg->block_sizes, cfg->n_block_sizes, K->nb));
    CPPHF_TRY(dm_check_nb(K->nb));
    CPPHF_TRY(check_mixed(K, cfg->mixed_switch_grad));
    const DmLayout L = dm_layout(K);
    if (!ws || wsb < L.total)
        return fail(CPPHF_ERR_INVALID, "solve_dm: workspace too small (" + std::to_string(L.total) + " bytes needed)");
    const SolveStream guard(st);
    st = guard.stream();
    // Not captured: projector callbacks (host round trips) and the superlattice
    // exchange, whose per-call channel tables are copied from host buffers that
    // a replayed graph would read after they are gone.
    const bool sl_path = K->sl && (K->sl->fock_active || K->sl->hartree_active);
    const bool use_graphs = cfg->graphs != 0 && guard.capturable && !project && !sl_path && solve_graphs_enabled();
    IterGraphs graphs;
    unsigned char* W = static_cast<unsigned char*>(ws);
    auto fld = [&](size_t off) { return reinterpret_cast<double2*>(W + off); };
    auto vec = [&](size_t off) { return reinterpret_cast<double*>(W + off); };
    double2 *Q = fld(L.Q), *P = fld(L.P), *Sig = fld(L.Sig), *F = fld(L.F), *Vd = fld(L.Vd);
    double2* G[2] = {fld(L.G[0]), fld(L.G[1])};
    double2* dQ[2] = {fld(L.dQ[0]), fld(L.dQ[1])};
    double *p = vec(L.p), *eps = vec(L.eps), *lam = vec(L.lam), *ew = vec(L.ew), *wn = vec(L.wn);
    double* g[2] = {vec(L.g[0]), vec(L.g[1])};
    double* dp[2] = {vec(L.dp[0]), vec(L.dp[1])};
    DmScalars* S = reinterpret_cast<DmScalars*>(W + L.S);
    void* fws = W + L.fock_ws;
    void* mws = W + L.mu_ws;

    const int64_t nk = K->nk1 * K->nk2;
    const int nb = (int)K->nb;
    const size_t fbytes = sizeof(double2) * (size_t)nk * nb * nb, vbytes = sizeof(double) * (size_t)nk * nb;
    const double wsum = std::max(K->weight_sum, TINY_REAL);
    const double n_t = n_e / wsum;
    const double T_r = std::max(K->T, 1.0e-12);
    const int64_t max_iter = std::max<int64_t>(0, cfg->max_iter);
    const int mu_it = cfg->mu_maxiter;

    CPPHF_CUDA(cudaMemsetAsync(S, 0, sizeof(DmScalars), st));
    k_scale_weights<<<grid_for(nk, 256), 256, 0, st>>>(K->w2d, wsum, wn, nk);
    CPPHF_LAUNCH_CHECK("scale weights");
    for (int b = 0; b < 2; ++b) {
        CPPHF_CUDA(cudaMemsetAsync(G[b], 0, fbytes, st));
        CPPHF_CUDA(cudaMemsetAsync(dQ[b], 0, fbytes, st));
        CPPHF_CUDA(cudaMemsetAsync(g[b], 0, vbytes, st));
        CPPHF_CUDA(cudaMemsetAsync(dp[b], 0, vbytes, st));
    }

    const bool small = dm_small_supported(nb);
    // density from (Q, occupations); small nb fuses p = expit((mu - ew)/T_r)
    auto density = [&](const double* ewv) -> int {
        if (small) {
            CPPHF_TRY(dm_small_dens_occ(Q, ewv, &S->mu, T_r, p, P, nk, nb, st));
        } else {
            CPPHF_TRY(dm_occupations(ewv, &S->mu, T_r, p, nk * nb, st));
            CPPHF_TRY(dm_density(Q, p, P, nk, nb, st));
        }
        if (project) {
            CPPHF_TRY(call_project(project, puser, P, K, st));
            CPPHF_TRY(hermitize(P, P, nk, nb, st));
        }
        return CPPHF_OK;
    };

    // ---- init (solver_dm.hpp:436-459) ----
    CPPHF_TRY(hermitize(P0, P, nk, nb, st));
    CPPHF_TRY(build_fock(K, P, Sig, F, nullptr, nullptr, nullptr, fws, L.fock_bytes, st));
    CPPHF_TRY(eigh_batched(F, ew, Q, nk, nb, 0, nullptr, st));
    CPPHF_TRY(mu_solve(ew, wn, nk, nb, n_t, &S->mu, T_r, mu_it, 1, &S->mu, mws, L.mu_bytes, st));

    double hbuf[4] = {0.0, 0.0, 0.0, 0.0};  // scalar read-back (pageable; each read is followed by a sync)

    double grad_norm = std::numeric_limits<double>::infinity();
    double E_prev = std::numeric_limits<double>::infinity();
    double dE = std::numeric_limits<double>::infinity();
    std::vector<double> hE((size_t)std::max<int64_t>(max_iter, 1)), hG((size_t)std::max<int64_t>(max_iter, 1));
    int64_t k = 0;
    const double fallback = std::pow(cfg->bt_shrink, (double)cfg->bt_max);
    // Switched precision: complex64 exchange until the gradient norm falls below
    // mixed_switch_grad (or the energy test would stop), then complex128.  The
    // plateau window and the CG restart count restart at the switch (k0).
    cpphf_kernel K32 = *K;
    K32.exchange_precision = 32;
    bool low = cfg->mixed_switch_grad > 0.0;
    int64_t k0 = 0;
    // One iteration (solver_dm.hpp:460-611): every launch, no host decision.
    auto iteration = [&](int cur, int prv, bool low_prec) -> int {
        const cpphf_kernel* Kb = low_prec ? &K32 : K;

        // 1. density (with occupations from the last eps_work and mu) + Fock + energy
        CPPHF_TRY(density(ew));
        CPPHF_TRY(build_fock(Kb, P, Sig, F, nullptr, &S->energy, nullptr, fws, L.fock_bytes, st));
        // 2.-4. Ft = Q^H F Q, gradient, preconditioner, PR+ direction
        if (small) {
            CPPHF_TRY(dm_small_rot_grad(Q, F, p, wn, eps, G[cur], g[cur], nk, nb, T_r, cfg->denom_scale, S, st));
            CPPHF_TRY(dm_small_pr_beta(G[cur], G[prv], g[cur], g[prv], eps, p, wn, nk, nb, T_r, (int)cfg->cg_restart,
                                       S, st));
            CPPHF_TRY(dm_small_direction(G[cur], dQ[prv], g[cur], dp[prv], eps, p, wn, dQ[cur], dp[cur], nk, nb, T_r,
                                         cfg->max_step, S, st));
        } else {
            CPPHF_TRY(dm_rotate(Q, F, F, eps, nk, nb, st));
            CPPHF_TRY(dm_gradient(F, p, eps, wn, G[cur], g[cur], nk, nb, T_r, cfg->denom_scale, S, st));
            CPPHF_TRY(dm_pr_beta(G[cur], G[prv], g[cur], g[prv], eps, p, wn, nk, nb, T_r, (int)cfg->cg_restart, S,
                                 st));
            CPPHF_TRY(dm_direction(G[cur], dQ[prv], g[cur], dp[prv], eps, p, wn, dQ[cur], dp[cur], nk, nb, T_r,
                                   cfg->max_step, S, st));
        }
        // 5. Cayley line search (elimination form of the spectral Cayley factor):
        // one pass per trial; a pass after the accepted trial returns at once
        for (int64_t bt = 0; bt < cfg->bt_max; ++bt) {
            if (small)
                CPPHF_TRY(dm_small_trial(dQ[cur], F, p, dp[cur], wn, ew, Vd, nk, nb, T_r, cfg->bt_shrink,
                                         bt == cfg->bt_max - 1, fallback, S, st));
            else
                CPPHF_TRY(dm_trial_lu(dQ[cur], F, p, dp[cur], wn, nk, nb, T_r, cfg->bt_shrink,
                                      bt == cfg->bt_max - 1, fallback, S, st));
        }
        // 6. retraction and mu (occupations are formed by the next density step)
        if (small)
            CPPHF_TRY(dm_small_retract(Q, dQ[cur], F, ew, Vd, nk, nb, S, st));
        else
            CPPHF_TRY(dm_retract_lu(Q, dQ[cur], F, ew, nk, nb, S, st));
        CPPHF_TRY(mu_solve(ew, wn, nk, nb, n_t, &S->mu, T_r, mu_it, 1, &S->mu, mws, L.mu_bytes, st));
        return CPPHF_OK;
    };
    while (k < max_iter) {
        bool e_nc;
        const int64_t kk = k - k0;
        if (cfg->plateau_window > 0 && kk > cfg->plateau_window) {
            e_nc = (hE[k - 1 - cfg->plateau_window] - hE[k - 1]) > cfg->tol_E;
        } else {
            e_nc = dE > cfg->tol_E;
        }
        const bool g_nc = (cfg->tol_grad > 0.0) && (grad_norm > cfg->tol_grad);
        if (low && (!(e_nc || g_nc) || grad_norm < cfg->mixed_switch_grad)) {
            low = false;
            k0 = k;
            CPPHF_CUDA(cudaMemsetAsync(&S->iter, 0, sizeof(int), st));
            dE = std::numeric_limits<double>::infinity();
            E_prev = std::numeric_limits<double>::infinity();
            continue;
        }
        if (!(e_nc || g_nc)) break;
        const int cur = (int)(k & 1), prv = cur ^ 1;
        IterGraphs& gr = graphs;
        const int lw = low ? 1 : 0;
        if (use_graphs && !gr.exec[cur][lw] && !gr.failed[cur][lw] && k - k0 >= 1) {
            // capture this parity and precision once (after an eager iteration
            // has set every kernel attribute); a failed capture runs eagerly
            cudaGraph_t g = nullptr;
            if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
                gr.failed[cur][lw] = true;
            } else {
                const int rc = iteration(cur, prv, low);
                const cudaError_t e = cudaStreamEndCapture(st, &g);
                if (rc != CPPHF_OK || e != cudaSuccess || !g ||
                    cudaGraphInstantiate(&gr.exec[cur][lw], g, 0) != cudaSuccess) {
                    gr.failed[cur][lw] = true;
                    gr.exec[cur][lw] = nullptr;
                }
                if (g) cudaGraphDestroy(g);
            }
            (void)cudaGetLastError();
        }
        if (gr.exec[cur][lw])
            CPPHF_CUDA(cudaGraphLaunch(gr.exec[cur][lw], st));
        else
            CPPHF_TRY(iteration(cur, prv, low));
        // 7. record: mu, mu_new, energy, grad_norm are adjacent in DmScalars (one copy)
        static_assert(offsetof(DmScalars, grad_norm) == offsetof(DmScalars, mu) + 3 * sizeof(double),
                      "DmScalars read-back layout");
        CPPHF_CUDA(cudaMemcpyAsync(hbuf, &S->mu, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CPPHF_CUDA(cudaStreamSynchronize(st));
        if (!std::isfinite(hbuf[0]))
            return fail(CPPHF_ERR_TIMEOUT, "solve_dm: chemical-potential solve failed (device wait timeout or non-finite)");
        const double E = hbuf[2];
        grad_norm = hbuf[3];
        hE[k] = E;
        hG[k] = grad_norm;
        dE = std::fabs(E - E_prev);
        E_prev = E;
        ++k;
    }

    // ---- finalize (solver_dm.hpp:615-652) ----
    CPPHF_TRY(density(ew));
    CPPHF_TRY(build_fock(K, P, Sig, F, nullptr, nullptr, nullptr, fws, L.fock_bytes, st));
    CPPHF_TRY(dm_rotate(Q, F, F, nullptr, nk, nb, st));
    CPPHF_TRY(eigh_batched(F, ew, Vd, nk, nb, 0, nullptr, st));
    CPPHF_TRY(dm_q_times_u(Q, Vd, nk, nb, st));
    CPPHF_TRY(mu_solve(ew, wn, nk, nb, n_t, &S->mu, T_r, mu_it, 1, &S->mu, mws, L.mu_bytes, st));
    CPPHF_TRY(density(ew));
    CPPHF_TRY(build_fock(K, P, Sig, F, nullptr, &S->energy, nullptr, fws, L.fock_bytes, st));
    if (Q_out) CPPHF_CUDA(cudaMemcpyAsync(Q_out, Q, fbytes, cudaMemcpyDeviceToDevice, st));
    if (p_out) CPPHF_CUDA(cudaMemcpyAsync(p_out, p, vbytes, cudaMemcpyDeviceToDevice, st));
    if (D_out) CPPHF_CUDA(cudaMemcpyAsync(D_out, P, fbytes, cudaMemcpyDeviceToDevice, st));
    if (F_out) CPPHF_CUDA(cudaMemcpyAsync(F_out, F, fbytes, cudaMemcpyDeviceToDevice, st));
    CPPHF_CUDA(cudaMemcpyAsync(hbuf, &S->energy, sizeof(double), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaMemcpyAsync(hbuf + 2, &S->mu, sizeof(double), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    if (!std::isfinite(hbuf[2]))
        return fail(CPPHF_ERR_TIMEOUT, "solve_dm: chemical-potential solve failed (device wait timeout or non-finite)");
    res->energy = hbuf[0];
    res->mu = hbuf[2];
    res->n_iter = k;
    res->converged = (k < max_iter) ? 1 : 0;
    for (int64_t i = 0; i < k; ++i) {
        if (hist_E) hist_E[i] = hE[i];
        if (hist_G) hist_G[i] = hG[i];
    }
    return CPPHF_OK;
}

// ---------------------------------------------------------------------------
// SCF
// ---------------------------------------------------------------------------
namespace {

struct ScfLayout {
    size_t D, Sig, F, Pn, V, eps, sh, occ, S, fock_ws, mu_ws, mu2, total;
    size_t fock_bytes, mu_bytes;
};

ScfLayout scf_layout(const cpphf_kernel* K) {
    const size_t nk = (size_t)K->nk1 * K->nk2, nb = (size_t)K->nb;
    const size_t fld = sizeof(double2) * nk * nb * nb, vec = sizeof(double) * nk * nb;
    SolverWs W;
    ScfLayout L;
    L.D = W.take(fld);
    L.Sig = W.take(fld);
    L.F = W.take(fld);
    L.Pn = W.take(fld);
    L.V = W.take(fld);
    L.eps = W.take(vec);
    L.sh = W.take(vec);
    L.occ = W.take(vec);
    L.mu2 = W.take(4 * sizeof(double));
    L.S = W.take(sizeof(DmScalars));
    L.fock_bytes = fock_bytes_any_precision(K);
    L.fock_ws = W.take(L.fock_bytes);
    L.mu_bytes = mu_workspace_bytes((int64_t)nk, (int64_t)nb);
    L.mu_ws = W.take(L.mu_bytes);
    L.total = W.total;
    return L;
}

}  // namespace

size_t solve_scf_workspace_bytes(const cpphf_kernel* K) { return scf_layout(K).total; }

int solve_scf(const cpphf_kernel* K, const cpphf_scf_config* cfg, const double2* P0, double n_e,
              cpphf_project_fn project, void* puser, double2* D_out, double2* F_out, double* hist_E, double* hist_D,
              double* hist_C, cpphf_scf_result* res, void* ws, size_t wsb, cudaStream_t st) {
    CPPHF_TRY(validate_kernel(K));
    if (!cfg || !P0 || !res) return fail(CPPHF_ERR_INVALID, "solve_scf: null argument");
    if (cfg->acceleration != 0)
        return fail(CPPHF_ERR_UNSUPPORTED, "SCF acceleration 'diis'/'oda' is not built into this library");
    CPPHF_TRY(dm_check_nb(K->nb));
    CPPHF_TRY(check_mixed(K, cfg->mixed_switch_tol));
    const ScfLayout L = scf_layout(K);
    if (!ws || wsb < L.total)
        return fail(CPPHF_ERR_INVALID, "solve_scf: workspace too small (" + std::to_string(L.total) + " bytes needed)");
    unsigned char* W = static_cast<unsigned char*>(ws);
    auto fld = [&](size_t off) { return reinterpret_cast<double2*>(W + off); };
    auto vec = [&](size_t off) { return reinterpret_cast<double*>(W + off); };
    double2 *D = fld(L.D), *Sig = fld(L.Sig), *F = fld(L.F), *Pn = fld(L.Pn), *V = fld(L.V);
    double *eps = vec(L.eps), *sh = vec(L.sh), *occ = vec(L.occ), *mu2 = vec(L.mu2);
    DmScalars* S = reinterpret_cast<DmScalars*>(W + L.S);
    void* fws = W + L.fock_ws;
    void* mws = W + L.mu_ws;
    const int64_t nk = K->nk1 * K->nk2;
    const int nb = (int)K->nb;
    const size_t fbytes = sizeof(double2) * (size_t)nk * nb * nb;
    const int64_t max_iter = std::max<int64_t>(0, cfg->max_iter);
    CPPHF_CUDA(cudaMemsetAsync(S, 0, sizeof(DmScalars), st));
    CPPHF_CUDA(cudaMemcpyAsync(D, P0, fbytes, cudaMemcpyDeviceToDevice, st));

    double hbuf[4] = {0.0, 0.0, 0.0, 0.0};  // scalar read-back (pageable; each read is followed by a sync)

    // switched precision: complex64 exchange until the density and commutator
    // residuals both fall below mixed_switch_tol; convergence is only accepted
    // in complex128
    cpphf_kernel K32 = *K;
    K32.exchange_precision = 32;
    bool low = cfg->mixed_switch_tol > 0.0;

    // the occupation mu: mu2[1] after a level shift, else mu2[0]
    double* mu_fin = (cfg->level_shift != 0.0) ? &mu2[1] : &mu2[0];
    // build_and_occupy (solver_scf.hpp:179-197); mu -> mu_fin, E -> S->energy
    // D is exactly Hermitian after the mixing kernel (it writes h and conj(h)) and
    // after a copy of P_new; hermitizing it again is a bitwise no-op and is skipped
    bool d_hermitian = false;
    auto build_and_occupy = [&]() -> int {
        if (project) CPPHF_TRY(call_project(project, puser, D, K, st));
        if (project || !d_hermitian) CPPHF_TRY(hermitize(D, D, nk, nb, st));
        CPPHF_TRY(build_fock(low ? &K32 : K, D, Sig, F, nullptr, &S->energy, nullptr, fws, L.fock_bytes, st));
        if (project) {
            CPPHF_TRY(call_project(project, puser, F, K, st));
            CPPHF_TRY(hermitize(F, F, nk, nb, st));
        }
        // density_from_fock (solver_scf.hpp:96-154)
        CPPHF_TRY(eigh_batched(F, eps, V, nk, nb, 0, nullptr, st));
        CPPHF_TRY(mu_solve(eps, K->w2d, nk, nb, n_e, nullptr, K->T, 30, 0, &mu2[0], mws, L.mu_bytes, st));
        const double* e_occ = eps;
        if (cfg->level_shift != 0.0) {
            k_level_shift<<<grid_for(nk * nb, 256), 256, 0, st>>>(eps, &mu2[0], K->T, cfg->level_shift, sh, nk * nb);
            CPPHF_LAUNCH_CHECK("level shift");
            e_occ = sh;
        }
        // without a level shift the second bisection (solver_scf.hpp:136) runs on an
        // unchanged copy of eps and returns mu_raw itself
        if (cfg->level_shift != 0.0)
            CPPHF_TRY(mu_solve(e_occ, K->w2d, nk, nb, n_e, nullptr, K->T, 30, 0, mu_fin, mws, L.mu_bytes, st));
        k_fermi<<<grid_for(nk * nb, 256), 256, 0, st>>>(e_occ, mu_fin, K->T, occ, nk * nb);
        CPPHF_LAUNCH_CHECK("fermi");
        // dm_density writes (X + X^H) / 2, exactly Hermitian: only a projector needs
        // the hermitisation again
        CPPHF_TRY(dm_density(V, occ, Pn, nk, nb, st));
        if (project) {
            CPPHF_TRY(call_project(project, puser, Pn, K, st));
            CPPHF_TRY(hermitize(Pn, Pn, nk, nb, st));
        }
        return CPPHF_OK;
    };

    bool converged = false;
    int64_t k = 0;
    const double wsum = std::max(K->weight_sum, 1.0e-30);
    const unsigned tgrid = [&] {
        const int64_t teams = nb <= kTeamWarpMaxNb ? kWarpTeams : 1;
        return (unsigned)std::max<int64_t>(1, std::min<int64_t>((nk + teams - 1) / teams, kDmMaxPartials));
    }();
    const bool warp = nb <= kTeamWarpMaxNb;
    const size_t per = (sizeof(double2) * team_mat_elems(nb) * 2 + 15) & ~(size_t)15;
    const size_t rsmem = per * (warp ? kWarpTeams : 1);
    static std::once_flag attrs;
    std::call_once(attrs, [] {
        raise_smem(k_scf_residuals<true>);
        raise_smem(k_scf_residuals<false>);
    });
    while (k < max_iter && !converged) {
        CPPHF_TRY(build_and_occupy());
        if (warp)
            k_scf_residuals<true><<<tgrid, 32 * kWarpTeams, rsmem, st>>>(F, D, Pn, K->w2d, nk, nb, S);
        else
            k_scf_residuals<false><<<tgrid, kCtaTeamThreadsDense, rsmem, st>>>(F, D, Pn, K->w2d, nk, nb, S);
        CPPHF_LAUNCH_CHECK("scf residuals");
        // energy, grad_norm (density residual) and lam_pc (commutator residual) are
        // adjacent in DmScalars: one copy, plus mu
        static_assert(offsetof(DmScalars, lam_pc) == offsetof(DmScalars, energy) + 2 * sizeof(double),
                      "DmScalars read-back layout");
        CPPHF_CUDA(cudaMemcpyAsync(hbuf, &S->energy, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CPPHF_CUDA(cudaMemcpyAsync(hbuf + 3, mu_fin, sizeof(double), cudaMemcpyDeviceToHost, st));
        CPPHF_CUDA(cudaStreamSynchronize(st));
        if (!std::isfinite(hbuf[3]))
            return fail(CPPHF_ERR_TIMEOUT, "solve_scf: chemical-potential solve failed (device wait timeout or non-finite)");
        const double d_res = std::sqrt(hbuf[1] / wsum);
        const double c_res = std::sqrt(hbuf[2] / wsum);
        converged = (d_res <= cfg->density_tol) && (c_res <= cfg->comm_tol);
        if (low && (converged || std::max(d_res, c_res) < cfg->mixed_switch_tol)) {
            // switch: mix as usual; the next build runs in complex128
            low = false;
            converged = false;
        }
        d_hermitian = true;
        if (converged) {
            CPPHF_CUDA(cudaMemcpyAsync(D, Pn, fbytes, cudaMemcpyDeviceToDevice, st));
        } else {
            k_scf_mix<<<grid_for(nk * (int64_t)nb * (nb + 1) / 2, 256), 256, 0, st>>>(D, Pn, cfg->mixing, nk, nb);
            CPPHF_LAUNCH_CHECK("scf mix");
            if (project) {
                CPPHF_TRY(call_project(project, puser, D, K, st));
                CPPHF_TRY(hermitize(D, D, nk, nb, st));
            }
        }
        if (hist_E) hist_E[k] = hbuf[0];
        if (hist_D) hist_D[k] = d_res;
        if (hist_C) hist_C[k] = c_res;
        ++k;
    }
    CPPHF_TRY(build_and_occupy());
    if (D_out) CPPHF_CUDA(cudaMemcpyAsync(D_out, D, fbytes, cudaMemcpyDeviceToDevice, st));
    if (F_out) CPPHF_CUDA(cudaMemcpyAsync(F_out, F, fbytes, cudaMemcpyDeviceToDevice, st));
    CPPHF_CUDA(cudaMemcpyAsync(hbuf, &S->energy, sizeof(double), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaMemcpyAsync(hbuf + 3, mu_fin, sizeof(double), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    if (!std::isfinite(hbuf[3]))
        return fail(CPPHF_ERR_TIMEOUT, "solve_scf: chemical-potential solve failed (device wait timeout or non-finite)");
    res->energy = hbuf[0];
    res->mu = hbuf[3];
    res->iterations = k;
    res->converged = converged ? 1 : 0;
    return CPPHF_OK;
}

// ---------------------------------------------------------------------------
// density_from_fock (solver_scf.hpp:96-154, dense eigh branch)
// ---------------------------------------------------------------------------
size_t density_from_fock_workspace_bytes(int64_t nk, int64_t nb) {
    SolverWs W;
    W.take(sizeof(double) * (size_t)nk * nb);  // shifted energies
    W.take(sizeof(double) * (size_t)nk * nb);  // occupations
    W.take(4 * sizeof(double));                // mu_raw, mu
    W.take(mu_workspace_bytes(nk, nb));
    return W.total;
}

int density_from_fock(const double2* F, const double* w, int64_t nk1, int64_t nk2, int64_t nb, double n_e, double T,
                      double level_shift, double2* P, double* eps, double2* V, double* mu_out, void* ws, size_t wsb,
                      cudaStream_t st) {
    if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(CPPHF_ERR_INVALID, "density_from_fock: empty mesh or nb");
    if (!F || !w || !P || !eps || !V || !mu_out) return fail(CPPHF_ERR_INVALID, "density_from_fock: null pointer");
    CPPHF_TRY(dm_check_nb(nb));
    const int64_t nk = nk1 * nk2;
    const size_t need = density_from_fock_workspace_bytes(nk, nb);
    if (!ws || wsb < need)
        return fail(CPPHF_ERR_INVALID, "density_from_fock: workspace too small (" + std::to_string(need) + " bytes needed)");
    SolverWs W;
    unsigned char* base = static_cast<unsigned char*>(ws);
    double* sh = reinterpret_cast<double*>(base + W.take(sizeof(double) * (size_t)nk * nb));
    double* occ = reinterpret_cast<double*>(base + W.take(sizeof(double) * (size_t)nk * nb));
    double* mu2 = reinterpret_cast<double*>(base + W.take(4 * sizeof(double)));
    const size_t mb = mu_workspace_bytes(nk, nb);
    void* mws = base + W.take(mb);
    CPPHF_TRY(eigh_batched(F, eps, V, nk, (int)nb, 0, nullptr, st));
    CPPHF_TRY(mu_solve(eps, w, nk, nb, n_e, nullptr, T, 30, 0, &mu2[0], mws, mb, st));
    const double* e_occ = eps;
    const double* mu = &mu2[0];
    if (level_shift != 0.0) {
        k_level_shift<<<grid_for(nk * nb, 256), 256, 0, st>>>(eps, &mu2[0], T, level_shift, sh, nk * nb);
        CPPHF_LAUNCH_CHECK("level shift");
        e_occ = sh;
        CPPHF_TRY(mu_solve(e_occ, w, nk, nb, n_e, nullptr, T, 30, 0, &mu2[1], mws, mb, st));
        mu = &mu2[1];
    }
    k_fermi<<<grid_for(nk * nb, 256), 256, 0, st>>>(e_occ, mu, T, occ, nk * nb);
    CPPHF_LAUNCH_CHECK("fermi");
    CPPHF_TRY(dm_density(V, occ, P, nk, (int)nb, st));
    CPPHF_CUDA(cudaMemcpyAsync(mu_out, mu, sizeof(double), cudaMemcpyDeviceToDevice, st));
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

size_t cpphf_density_from_fock_workspace_bytes(int64_t nk, int64_t nb) {
    return cpphf::density_from_fock_workspace_bytes(nk, nb);
}

int cpphf_density_from_fock(const void* F, const double* w, int64_t nk1, int64_t nk2, int64_t nb, double n_e,
                            double T, double level_shift, void* P, double* eps, void* V, double* mu, void* workspace,
                            size_t workspace_bytes, void* stream) {
    return cpphf::density_from_fock(static_cast<const double2*>(F), w, nk1, nk2, nb, n_e, T, level_shift,
                                    static_cast<double2*>(P), eps, static_cast<double2*>(V), mu, workspace,
                                    workspace_bytes, static_cast<cudaStream_t>(stream));
}

size_t cpphf_solve_dm_workspace_bytes(const cpphf_kernel* K) { return K ? cpphf::solve_dm_workspace_bytes(K) : 0; }

int cpphf_solve_dm(const cpphf_kernel* K, const cpphf_dm_config* cfg, const void* P0, double n_e,
                   cpphf_project_fn project, void* project_user, void* Q_out, double* p_out, void* density_out,
                   void* fock_out, double* hist_E, double* hist_grad, cpphf_dm_result* result, void* workspace,
                   size_t workspace_bytes, void* stream) {
    return cpphf::solve_dm(K, cfg, static_cast<const double2*>(P0), n_e, project, project_user,
                           static_cast<double2*>(Q_out), p_out, static_cast<double2*>(density_out),
                           static_cast<double2*>(fock_out), hist_E, hist_grad, result, workspace, workspace_bytes,
                           static_cast<cudaStream_t>(stream));
}

size_t cpphf_solve_scf_workspace_bytes(const cpphf_kernel* K) { return K ? cpphf::solve_scf_workspace_bytes(K) : 0; }

int cpphf_solve_scf(const cpphf_kernel* K, const cpphf_scf_config* cfg, const void* P0, double n_e,
                    cpphf_project_fn project, void* project_user, void* density_out, void* fock_out,
                    double* hist_E, double* hist_density, double* hist_comm, cpphf_scf_result* result,
                    void* workspace, size_t workspace_bytes, void* stream) {
    return cpphf::solve_scf(K, cfg, static_cast<const double2*>(P0), n_e, project, project_user,
                            static_cast<double2*>(density_out), static_cast<double2*>(fock_out), hist_E, hist_density,
                            hist_comm, result, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
