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
#include "rtr.cuh"
#include "solve_util.cuh"
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
                                DmScalars* S, double2* __restrict__ comm_out) {
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
            if (comm_out) comm_out[(size_t)k * nb * nb + e] = c;
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
__global__ void k_scf_mix(const double2* D, const double2* Pn, double mixing, double2* out, int64_t nk, int nb) {
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
        const double2 a = scf_mix_elem(dij, Pn[ij], mixing);
        const double2 b = scf_mix_elem(dji, Pn[ji], mixing);
        const double2 h = scf_mix_herm(a, b);
        out[ij] = h;
        out[ji] = cconj(h);
    }
}

// ---------------------------------------------------------------------------
// SCF acceleration (solver_scf.hpp:253-428)
// ---------------------------------------------------------------------------
constexpr int kDiisMax = 16;  // history slots a launch handles

struct FieldSet {
    const double2* p[kDiisMax];
};

// out[i] = sum_k w_k Re sum_a conj(H_i[k, a]) Rn[k, a] for the m history
// residuals H_i (the new row of the C-DIIS matrix B, solver_scf.hpp:273-289)
__global__ void k_diis_dots(FieldSet H, int m, const double2* __restrict__ Rn, const double* __restrict__ w,
                            int64_t nk, int nb2, DmScalars* S, double* __restrict__ out) {
    __shared__ double red[32 * kDiisMax];
    double v[kDiisMax];
#pragma unroll
    for (int i = 0; i < kDiisMax; ++i) v[i] = 0.0;
    const int64_t n = nk * nb2;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double wk = w[e / nb2];
        const double2 r = Rn[e];
#pragma unroll
        for (int i = 0; i < kDiisMax; ++i) {
            if (i < m) {
                const double2 a = H.p[i][e];
                v[i] += wk * (a.x * r.x + a.y * r.y);
            }
        }
    }
    double o[kDiisMax];
    if (reduce_last_block<kDiisMax>(v, S->part, &S->counter, o, red) && threadIdx.x == 0)
        for (int i = 0; i < m; ++i) out[i] = o[i];
}

// Fex = damp sum_i c_i F_i + (1 - damp) Fcur, summed in history order
// (solver_scf.hpp:305-320); the caller hermitizes
struct DiisCoef {
    double c[kDiisMax];
};
__global__ void k_diis_extrapolate(FieldSet Fh, DiisCoef cf, int m, double damp, const double2* __restrict__ Fcur,
                                   double2* __restrict__ Fex, int64_t n) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = mk(0.0, 0.0);
#pragma unroll
        for (int i = 0; i < kDiisMax; ++i) {
            if (i < m) {
                const double2 f = Fh.p[i][e];
                acc = mk(acc.x + cf.c[i] * f.x, acc.y + cf.c[i] * f.y);
            }
        }
        if (damp < 1.0) {
            const double2 f = Fcur[e];
            acc = mk(damp * acc.x + (1.0 - damp) * f.x, damp * acc.y + (1.0 - damp) * f.y);
        }
        Fex[e] = acc;
    }
}

// c1 = sum_k w_k Re tr(F_k (Pn_k - D_k)) (ODA slope, solver_scf.hpp:362-374)
__global__ void k_oda_c1(const double2* __restrict__ F, const double2* __restrict__ D, const double2* __restrict__ Pn,
                         const double* __restrict__ w, int64_t nk, int nb, DmScalars* S, double* __restrict__ out) {
    __shared__ double red[32];
    double v[1] = {0.0};
    const int nb2 = nb * nb;
    const int64_t n = nk * nb2;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / nb2;
        const int r = (int)(e - k * nb2), a = r / nb, b = r - a * nb;
        const size_t ba = (size_t)k * nb2 + (size_t)b * nb + a;
        const double2 f = F[e];
        const double2 d = csub(Pn[ba], D[ba]);
        v[0] += w[k] * (f.x * d.x - f.y * d.y);
    }
    double o[1];
    if (reduce_last_block<1>(v, S->part, &S->counter, o, red) && threadIdx.x == 0) *out = o[0];
}

// sum_k w_k ||A_k - B_k||_F^2 (weighted_difference_norm before its division,
// solver_scf.hpp:77-91)
__global__ void k_wdiff2(const double2* __restrict__ A, const double2* __restrict__ B, const double* __restrict__ w,
                         int64_t nk, int nb2, DmScalars* S, double* __restrict__ out) {
    __shared__ double red[32];
    double v[1] = {0.0};
    const int64_t n = nk * nb2;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 d = csub(A[e], B[e]);
        v[0] += w[e / nb2] * (d.x * d.x + d.y * d.y);
    }
    double o[1];
    if (reduce_last_block<1>(v, S->part, &S->counter, o, red) && threadIdx.x == 0) *out = o[0];
}

// Solve [B -1; -1^T 0] [c; l] = [0; -1] (size n = m + 1, row-major A) by
// Gaussian elimination with complete pivoting.  False when the matrix is
// rank-deficient at the threshold of Eigen's FullPivLU::isInvertible (a pivot
// below eps * n * |first pivot|, the reference's check, solver_scf.hpp:291-300)
// or the solution is not finite.
bool diis_solve(std::vector<double> A, int n, std::vector<double>& x) {
    std::vector<double> b((size_t)n, 0.0);
    b[(size_t)n - 1] = -1.0;
    std::vector<int> colp((size_t)n);
    for (int i = 0; i < n; ++i) colp[(size_t)i] = i;
    double maxpiv = 0.0;
    const double thr = std::numeric_limits<double>::epsilon() * n;
    for (int kk = 0; kk < n; ++kk) {
        int pr = kk, pc = kk;
        double best = -1.0;
        for (int i = kk; i < n; ++i)
            for (int j = kk; j < n; ++j)
                if (std::fabs(A[(size_t)i * n + j]) > best) {
                    best = std::fabs(A[(size_t)i * n + j]);
                    pr = i;
                    pc = j;
                }
        if (kk == 0) maxpiv = best;
        if (!(best > thr * maxpiv) || best == 0.0) return false;
        if (pr != kk) {
            for (int j = 0; j < n; ++j) std::swap(A[(size_t)kk * n + j], A[(size_t)pr * n + j]);
            std::swap(b[(size_t)kk], b[(size_t)pr]);
        }
        if (pc != kk) {
            for (int i = 0; i < n; ++i) std::swap(A[(size_t)i * n + kk], A[(size_t)i * n + pc]);
            std::swap(colp[(size_t)kk], colp[(size_t)pc]);
        }
        const double piv = A[(size_t)kk * n + kk];
        for (int i = kk + 1; i < n; ++i) {
            const double f = A[(size_t)i * n + kk] / piv;
            if (f == 0.0) continue;
            for (int j = kk; j < n; ++j) A[(size_t)i * n + j] -= f * A[(size_t)kk * n + j];
            b[(size_t)i] -= f * b[(size_t)kk];
        }
    }
    std::vector<double> y((size_t)n);
    for (int i = n - 1; i >= 0; --i) {
        double acc = b[(size_t)i];
        for (int j = i + 1; j < n; ++j) acc -= A[(size_t)i * n + j] * y[(size_t)j];
        y[(size_t)i] = acc / A[(size_t)i * n + i];
    }
    x.assign((size_t)n, 0.0);
    for (int i = 0; i < n; ++i) x[(size_t)colp[(size_t)i]] = y[(size_t)i];
    for (int i = 0; i < n - 1; ++i)
        if (!std::isfinite(x[(size_t)i])) return false;
    return true;
}

}  // namespace

namespace {
struct PinnedScalars {
    double* p = nullptr;
    ~PinnedScalars() {
        if (p) cudaFreeHost(p);
    }
};
}  // namespace

double* host_scalars() {
    thread_local PinnedScalars h;
    thread_local double pageable[kHostScalars];
    if (!h.p && cudaHostAlloc(reinterpret_cast<void**>(&h.p), kHostScalars * sizeof(double), cudaHostAllocDefault) !=
                    cudaSuccess) {
        (void)cudaGetLastError();
        h.p = nullptr;
        return pageable;
    }
    return h.p;
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

int scale_weights(const double* w, double wsum, double* out, int64_t n, cudaStream_t st) {
    k_scale_weights<<<grid_for(n, 256), 256, 0, st>>>(w, wsum, out, n);
    CPPHF_LAUNCH_CHECK("scale weights");
    return CPPHF_OK;
}

namespace {

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
    return std::max(fock_bytes_packed_kernel(K), fock_bytes_packed_kernel(&K32));
}

// Exchange precision of a switched solve: complex64 first, complex128 after.
int check_mixed(const cpphf_kernel* K, double sw) {
    if (!(sw >= 0.0)) return fail(CPPHF_ERR_INVALID, "mixed-precision switch threshold must be >= 0");
    if (sw > 0.0 && K->exchange_precision != 64)
        return fail(CPPHF_ERR_INVALID, "a switched-precision solve needs exchange_precision 64 in the kernel");
    return CPPHF_OK;
}

struct DmLayout {
    size_t Q, P, Sig, F, G[2], dQ[2], Vd, p, eps, g[2], dp[2], lam, ew, wn, S, fock_ws, mu_ws, pack, blk, total;
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
    L.pack = W.take(solver_pack_bytes(K));
    L.blk = W.take(2 * sizeof(unsigned long long));
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

// solver_dm.hpp:100-115: the block path needs no projector and h, refP and the
// active contact operators all block-diagonal in the given blocks.
int block_problem_invariant(const cpphf_kernel* K, bool project, const BlockSpec& bs, unsigned long long* dev2,
                            cudaStream_t st, bool* ok) {
    *ok = false;
    if (project) return CPPHF_OK;
    const int64_t nk = K->nk1 * K->nk2, nb = K->nb;
    bool good = false;
    CPPHF_TRY(block_structure_ok(static_cast<const double2*>(K->h), nk, nb, bs, dev2, st, &good));
    if (!good) return CPPHF_OK;
    if (K->has_refP) {
        CPPHF_TRY(block_structure_ok(static_cast<const double2*>(K->refP), nk, nb, bs, dev2, st, &good));
        if (!good) return CPPHF_OK;
    }
    if (K->contact_g && K->n_contact > 0 && K->contact_Oi && K->contact_Oj) {
        std::vector<double> g((size_t)K->n_contact);
        CPPHF_CUDA(cudaMemcpyAsync(g.data(), K->contact_g, sizeof(double) * g.size(), cudaMemcpyDeviceToHost, st));
        CPPHF_CUDA(cudaStreamSynchronize(st));
        for (int64_t t = 0; t < K->n_contact; ++t) {
            if (g[(size_t)t] == 0.0) continue;
            const double2* Oi = static_cast<const double2*>(K->contact_Oi) + t * nb * nb;
            const double2* Oj = static_cast<const double2*>(K->contact_Oj) + t * nb * nb;
            CPPHF_TRY(block_structure_ok(Oi, 1, nb, bs, dev2, st, &good));
            if (!good) return CPPHF_OK;
            CPPHF_TRY(block_structure_ok(Oj, 1, nb, bs, dev2, st, &good));
            if (!good) return CPPHF_OK;
        }
    }
    *ok = true;
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

}  // namespace

size_t solve_dm_workspace_bytes(const cpphf_kernel* K) { return dm_layout(K).total; }

int solve_dm(const cpphf_kernel* K, const cpphf_dm_config* cfg, const double2* P0, double n_e,
             cpphf_project_fn project, void* puser, double2* Q_out, double* p_out, double2* D_out, double2* F_out,
             double* hist_E, double* hist_G, cpphf_dm_result* res, void* ws, size_t wsb, cudaStream_t st) {
    CPPHF_TRY(validate_kernel(K));
    if (!cfg || !P0 || !res) return fail(CPPHF_ERR_INVALID, "solve_dm: null argument");
    if (cfg->optimizer == 1)  // cpp_hf_native.cpp:557-559: 1 is Newton, any other code the CG solver
        return solve_rtr(K, cfg, P0, n_e, project, puser, Q_out, p_out, D_out, F_out, hist_E, hist_G, res, ws, wsb,
                         st);
    CPPHF_TRY(check_block_sizes(cfg->block_sizes, cfg->n_block_sizes, K->nb));
    CPPHF_TRY(dm_check_nb(K->nb));
    CPPHF_TRY(check_mixed(K, cfg->mixed_switch_grad));
    const DmLayout L = dm_layout(K);
    if (!ws || wsb < L.total)
        return fail(CPPHF_ERR_INVALID, "solve_dm: workspace too small (" + std::to_string(L.total) + " bytes needed)");
    const SolveStream guard(st);
    st = guard.stream();
    cpphf_kernel Kp;  // K with its packed VR / h (Hermitian packing), made once per solve
    CPPHF_TRY(solver_pack(K, &Kp, static_cast<unsigned char*>(ws) + L.pack, st));
    K = &Kp;
    // Not captured: host projector callbacks (host round trips) and the superlattice
    // exchange, whose per-call channel tables are copied from host buffers that
    // a replayed graph would read after they are gone.
    const bool sl_path = K->sl && (K->sl->fock_active || K->sl->hartree_active);
    const bool use_graphs = cfg->graphs != 0 && guard.capturable && (!project || cfg->project_device != 0) &&
                            !sl_path;
    IterGraphs graphs;
    unsigned char* W = static_cast<unsigned char*>(ws);
    auto fld = [&](size_t off) { return reinterpret_cast<double2*>(W + off); };
    auto vec = [&](size_t off) { return reinterpret_cast<double*>(W + off); };
    double2 *Q = fld(L.Q), *P = fld(L.P), *Sig = fld(L.Sig), *F = fld(L.F), *Vd = fld(L.Vd);
    double2* G[2] = {fld(L.G[0]), fld(L.G[1])};
    double2* dQ[2] = {fld(L.dQ[0]), fld(L.dQ[1])};
    double *p = vec(L.p), *eps = vec(L.eps), *lam = vec(L.lam), *ew = vec(L.ew), *wn = vec(L.wn);
    double* ew2 = reinterpret_cast<double*>(Vd);  // second trial's eps_work (Vd is free inside the loop)
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

    // block-diagonal fast path (solver_dm.hpp:403-405): block eigh, eigenvalues
    // block by block, at the start and in the final polish; the elimination form
    // of the Cayley factor keeps the blocks of d in every trial and retraction
    BlockSpec bspec;
    bool use_block = false;
    unsigned long long* blk = reinterpret_cast<unsigned long long*>(W + L.blk);
    if (cfg->n_block_sizes > 1) {
        CPPHF_TRY(make_block_spec(nb, cfg->block_sizes, cfg->n_block_sizes, 0, bspec));
        CPPHF_TRY(block_problem_invariant(K, project != nullptr, bspec, blk, st, &use_block));
    }

    // ---- init (solver_dm.hpp:436-459) ----
    CPPHF_TRY(hermitize(P0, P, nk, nb, st));
    CPPHF_TRY(build_fock(K, P, solver_sigma(K, Sig), F, nullptr, nullptr, nullptr, fws, L.fock_bytes, st));
    if (use_block) CPPHF_TRY(block_structure_ok(F, nk, nb, bspec, blk, st, &use_block));
    CPPHF_TRY(eigh_batched(F, ew, Q, nk, nb, 0, use_block ? &bspec : nullptr, st));
    CPPHF_TRY(mu_solve(ew, wn, nk, nb, n_t, &S->mu, T_r, mu_it, 1, &S->mu, mws, L.mu_bytes, st));

    double* const hbuf = host_scalars();  // scalar read-back; each read is followed by a sync
    for (int i = 0; i < 4; ++i) hbuf[i] = 0.0;

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
        CPPHF_TRY(build_fock(Kb, P, solver_sigma(Kb, Sig), F, nullptr, &S->energy, nullptr, fws, L.fock_bytes, st));
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
        // small nb, two trials per pass; otherwise one pass per trial; a pass
        // after the accepted trial returns at once
        if (small) {
            // the factors U go to G[prv] and dQ[prv], which this iteration no
            // longer reads (PR+ and the direction are done; the next iteration
            // writes both before reading them)
            for (int64_t bt = 0; bt < cfg->bt_max; bt += 2)
                CPPHF_TRY(dm_small_trial2(dQ[cur], F, p, dp[cur], wn, ew, ew2, G[prv], dQ[prv], nk, nb, T_r,
                                          cfg->bt_shrink, (int)bt, (int)cfg->bt_max, fallback, S, st));
        } else {
            for (int64_t bt = 0; bt < cfg->bt_max; ++bt)
                CPPHF_TRY(dm_trial_lu(dQ[cur], F, p, dp[cur], wn, nk, nb, T_r, cfg->bt_shrink,
                                      bt == cfg->bt_max - 1, fallback, S, st));
        }
        // 6. retraction and mu (occupations are formed by the next density step)
        if (small)
            CPPHF_TRY(dm_small_retract(Q, dQ[cur], F, ew, ew2, G[prv], dQ[prv], nk, nb, S, st));
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
    CPPHF_TRY(build_fock(K, P, solver_sigma(K, Sig), F, nullptr, nullptr, nullptr, fws, L.fock_bytes, st));
    CPPHF_TRY(dm_rotate(Q, F, F, nullptr, nk, nb, st));
    CPPHF_TRY(eigh_batched(F, ew, Vd, nk, nb, 0, use_block ? &bspec : nullptr, st));
    CPPHF_TRY(dm_q_times_u(Q, Vd, nk, nb, st));
    CPPHF_TRY(mu_solve(ew, wn, nk, nb, n_t, &S->mu, T_r, mu_it, 1, &S->mu, mws, L.mu_bytes, st));
    CPPHF_TRY(density(ew));
    CPPHF_TRY(build_fock(K, P, solver_sigma(K, Sig), F, nullptr, &S->energy, nullptr, fws, L.fock_bytes, st));
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
    size_t D, Sig, F, Pn, V, eps, sh, occ, S, fock_ws, mu_ws, mu2, pack, blk, total;
    size_t fock_bytes, mu_bytes;
    size_t R, Fh, Fex, dots, Sn, Fn, Dpre;  // acceleration extras (0 when unused)
    int nhist;
};

// cfg == null: linear mixing without a trust radius
ScfLayout scf_layout(const cpphf_kernel* K, const cpphf_scf_config* cfg = nullptr) {
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
    L.R = L.Fh = L.Fex = L.dots = L.Sn = L.Fn = L.Dpre = 0;
    L.nhist = 0;
    if (cfg && cfg->acceleration == 1) {
        L.nhist = std::max(1, std::min<int>(cfg->diis_size, kDiisMax));
        L.R = W.take(fld * (size_t)L.nhist);
        L.Fh = W.take(fld * (size_t)L.nhist);
        L.Fex = W.take(fld);
        L.dots = W.take(sizeof(double) * kDiisMax);
    }
    if (cfg && cfg->acceleration == 2) {
        L.Sn = W.take(fld);
        L.Fn = W.take(fld);
    }
    if (cfg && cfg->trust_radius > 0.0) L.Dpre = W.take(fld);
    L.pack = W.take(solver_pack_bytes(K));
    L.blk = W.take(2 * sizeof(unsigned long long));
    L.total = W.total;
    return L;
}

}  // namespace

size_t solve_scf_workspace_bytes(const cpphf_kernel* K) { return scf_layout(K).total; }
size_t solve_scf_workspace_bytes_cfg(const cpphf_kernel* K, const cpphf_scf_config* cfg) {
    return scf_layout(K, cfg).total;
}

int solve_scf(const cpphf_kernel* K, const cpphf_scf_config* cfg, const double2* P0, double n_e,
              cpphf_project_fn project, void* puser, double2* D_out, double2* F_out, double* hist_E, double* hist_D,
              double* hist_C, cpphf_scf_result* res, void* ws, size_t wsb, cudaStream_t st) {
    CPPHF_TRY(validate_kernel(K));
    if (!cfg || !P0 || !res) return fail(CPPHF_ERR_INVALID, "solve_scf: null argument");
    if (cfg->acceleration < 0 || cfg->acceleration > 2)
        return fail(CPPHF_ERR_INVALID, "SCFConfig.acceleration must be 'linear', 'diis', or 'oda'");
    if (cfg->acceleration == 1 && cfg->diis_size < 1) return fail(CPPHF_ERR_INVALID, "SCF diis_size must be positive");
    if (cfg->acceleration == 1 && cfg->diis_size > kDiisMax)
        return fail(CPPHF_ERR_UNSUPPORTED, "SCF diis_size above " + std::to_string(kDiisMax) + " is not supported");
    CPPHF_TRY(dm_check_nb(K->nb));
    CPPHF_TRY(check_mixed(K, cfg->mixed_switch_tol));
    const ScfLayout L = scf_layout(K, cfg);
    if (!ws || wsb < L.total)
        return fail(CPPHF_ERR_INVALID, "solve_scf: workspace too small (" + std::to_string(L.total) + " bytes needed)");
    const SolveStream guard(st);
    st = guard.stream();
    cpphf_kernel Kp;  // K with its packed VR / h (Hermitian packing), made once per solve
    CPPHF_TRY(solver_pack(K, &Kp, static_cast<unsigned char*>(ws) + L.pack, st));
    K = &Kp;
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

    double* const hbuf = host_scalars();  // scalar read-back; each read is followed by a sync
    for (int i = 0; i < 4; ++i) hbuf[i] = 0.0;

    // switched precision: complex64 exchange until the density and commutator
    // residuals both fall below mixed_switch_tol; convergence is only accepted
    // in complex128
    cpphf_kernel K32 = *K;
    K32.exchange_precision = 32;
    bool low = cfg->mixed_switch_tol > 0.0;

    // block-diagonal eigh in density_from_fock (solver_scf.hpp:96-124): with more
    // than one block summing to nb, every F that is block-diagonal to 1e-10 of
    // its largest entry takes the block eigh (checked on each call, on the host)
    BlockSpec sbspec;
    bool scf_block = false;
    unsigned long long* blk = reinterpret_cast<unsigned long long*>(W + L.blk);
    if (cfg->block_sizes && cfg->n_block_sizes > 1) {
        int64_t tot = 0;
        bool pos = true;
        for (int64_t b = 0; b < cfg->n_block_sizes; ++b) {
            tot += cfg->block_sizes[b];
            pos = pos && cfg->block_sizes[b] > 0;
        }
        if (tot == nb && pos) {
            CPPHF_TRY(make_block_spec(nb, cfg->block_sizes, cfg->n_block_sizes, 0, sbspec));
            scf_block = true;
        }
    }

    // the occupation mu: mu2[1] after a level shift, else mu2[0]
    double* mu_fin = (cfg->level_shift != 0.0) ? &mu2[1] : &mu2[0];
    CPPHF_CUDA(cudaMemsetAsync(mu2, 0xFF, 2 * sizeof(double), st));  // NaN: no warm start yet
    // build_and_occupy (solver_scf.hpp:179-197); mu -> mu_fin, E -> S->energy
    // D is exactly Hermitian after the mixing kernel (it writes h and conj(h)) and
    // after a copy of P_new; hermitizing it again is a bitwise no-op and is skipped
    bool d_hermitian = false;
    // density_from_fock (solver_scf.hpp:96-154): P_out = herm(V f V^H) from Fsrc
    auto occupy = [&](const double2* Fsrc, double2* Pout) -> int {
        const BlockSpec* bsp = nullptr;
        if (scf_block) {
            bool ok = false;
            CPPHF_TRY(block_structure_ok(Fsrc, nk, nb, sbspec, blk, st, &ok));
            if (ok) bsp = &sbspec;
        }
        CPPHF_TRY(eigh_batched(Fsrc, eps, V, nk, nb, 0, bsp, st));
        // the previous iteration's mu warm-starts the bisection's root (same result)
        CPPHF_TRY(mu_solve(eps, K->w2d, nk, nb, n_e, &mu2[0], K->T, 30, 0, &mu2[0], mws, L.mu_bytes, st));
        const double* e_occ = eps;
        if (cfg->level_shift != 0.0) {
            k_level_shift<<<grid_for(nk * nb, 256), 256, 0, st>>>(eps, &mu2[0], K->T, cfg->level_shift, sh, nk * nb);
            CPPHF_LAUNCH_CHECK("level shift");
            e_occ = sh;
        }
        // without a level shift the second bisection (solver_scf.hpp:136) runs on an
        // unchanged copy of eps and returns mu_raw itself
        if (cfg->level_shift != 0.0)
            CPPHF_TRY(mu_solve(e_occ, K->w2d, nk, nb, n_e, mu_fin, K->T, 30, 0, mu_fin, mws, L.mu_bytes, st));
        // the density pass writes (X + X^H) / 2, exactly Hermitian: only a projector
        // needs the hermitisation again
        if (dm_small_supported(nb)) {
            // occupations expit((mu - e) / (T + 1e-12)) formed inside the density pass:
            // the same value as k_fermi's expit(-(e - mu) / (T + 1e-12)), one launch less
            CPPHF_TRY(dm_small_dens_occ(V, e_occ, mu_fin, K->T + 1.0e-12, occ, Pout, nk, nb, st));
        } else {
            k_fermi<<<grid_for(nk * nb, 256), 256, 0, st>>>(e_occ, mu_fin, K->T, occ, nk * nb);
            CPPHF_LAUNCH_CHECK("fermi");
            CPPHF_TRY(dm_density(V, occ, Pout, nk, nb, st));
        }
        if (project) {
            CPPHF_TRY(call_project(project, puser, Pout, K, st));
            CPPHF_TRY(hermitize(Pout, Pout, nk, nb, st));
        }
        return CPPHF_OK;
    };
    auto build_and_occupy = [&]() -> int {
        if (project) CPPHF_TRY(call_project(project, puser, D, K, st));
        if (project || !d_hermitian) CPPHF_TRY(hermitize(D, D, nk, nb, st));
        CPPHF_TRY(build_fock(low ? &K32 : K, D, solver_sigma(low ? &K32 : K, Sig), F, nullptr, &S->energy, nullptr, fws, L.fock_bytes, st));
        if (project) {
            CPPHF_TRY(call_project(project, puser, F, K, st));
            CPPHF_TRY(hermitize(F, F, nk, nb, st));
        }
        return occupy(F, Pn);
    };
    // density <- herm(A + s (B - A)), then the projector
    auto mix_into_D = [&](const double2* A, const double2* B, double s_) -> int {
        k_scf_mix<<<grid_for(nk * (int64_t)nb * (nb + 1) / 2, 256), 256, 0, st>>>(A, B, s_, D, nk, nb);
        CPPHF_LAUNCH_CHECK("scf mix");
        if (project) {
            CPPHF_TRY(call_project(project, puser, D, K, st));
            CPPHF_TRY(hermitize(D, D, nk, nb, st));
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

    // acceleration state
    const int acc = cfg->acceleration;
    const int64_t nel = nk * (int64_t)nb * nb;
    const int nb2 = nb * nb;
    const unsigned egrid = grid_for(nel, 256);
    // reductions with up to kDiisMax values per block must fit S->part
    const unsigned rgrid = std::min<unsigned>(egrid, (unsigned)((3 * kDmMaxPartials) / kDiisMax));
    double2* Rh = acc == 1 ? fld(L.R) : nullptr;
    double2* Fh = acc == 1 ? fld(L.Fh) : nullptr;
    double2* Fex = acc == 1 ? fld(L.Fex) : nullptr;
    double* dots = acc == 1 ? reinterpret_cast<double*>(W + L.dots) : nullptr;
    double2* Sn = acc == 2 ? fld(L.Sn) : nullptr;
    double2* Fn = acc == 2 ? fld(L.Fn) : nullptr;
    double2* Dpre = cfg->trust_radius > 0.0 ? fld(L.Dpre) : nullptr;
    const int nh = L.nhist;
    int hcount = 0, hhead = 0;  // DIIS ring: entries held, next slot
    // Bs[a * kDiisMax + b] = <R_a, R_b>_w for ring slots a, b
    std::vector<double> Bs((size_t)kDiisMax * kDiisMax, 0.0);
    double* const dbuf = hbuf + 8;  // DIIS overlaps of the newest residual
    static_assert(8 + kDiisMax + 3 <= kHostScalars, "host scalar layout");

    // Linear mixing without a projector, trust radius or superlattice terms: the
    // mix decided at the end of an iteration is deferred to the start of the next
    // one, so every iteration after the first is the same launch sequence (mix,
    // Fock build, occupations, residuals), captured once per precision.
    const bool sl_path = K->sl && (K->sl->fock_active || K->sl->hartree_active);
    const bool scf_graphs =
        cfg->graphs != 0 && guard.capturable && acc == 0 && !project && !Dpre && !sl_path && !scf_block;
    // On that path with nb <= 8 the residual pass also writes the mix into D (the
    // residuals need the unmixed D only in the same pass; a converged iteration
    // overwrites D with P_new), so no separate mix runs.
    const bool fuse_mix = scf_graphs && dm_small_supported(nb);
    IterGraphs sgr;
    bool pending_mix = false;
    while (k < max_iter && !converged) {
        double2* comm_out = acc == 1 ? Rh + (size_t)hhead * nel : nullptr;
        auto body = [&]() -> int {
            if (pending_mix) CPPHF_TRY(mix_into_D(D, Pn, cfg->mixing));
            CPPHF_TRY(build_and_occupy());
            // the new C-DIIS residual goes to the slot after the newest entry
            // (overwriting the oldest when the ring is full)
            if (dm_small_supported(nb))
                CPPHF_TRY(scf_small_residuals(F, D, Pn, K->w2d, nk, nb, S, comm_out, fuse_mix ? D : nullptr,
                                              cfg->mixing, st));
            else if (warp)
                k_scf_residuals<true><<<tgrid, 32 * kWarpTeams, rsmem, st>>>(F, D, Pn, K->w2d, nk, nb, S, comm_out);
            else
                k_scf_residuals<false><<<tgrid, kCtaTeamThreadsDense, rsmem, st>>>(F, D, Pn, K->w2d, nk, nb, S,
                                                                                    comm_out);
            CPPHF_LAUNCH_CHECK("scf residuals");
            return CPPHF_OK;
        };
        const int lw = low ? 1 : 0;
        bool replayed = false;
        if (scf_graphs && (pending_mix || fuse_mix) && d_hermitian) {
            if (!sgr.exec[0][lw] && !sgr.failed[0][lw]) {
                cudaGraph_t g = nullptr;
                if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
                    sgr.failed[0][lw] = true;
                } else {
                    const int rc = body();
                    const cudaError_t e = cudaStreamEndCapture(st, &g);
                    if (rc != CPPHF_OK || e != cudaSuccess || !g ||
                        cudaGraphInstantiate(&sgr.exec[0][lw], g, 0) != cudaSuccess) {
                        sgr.failed[0][lw] = true;
                        sgr.exec[0][lw] = nullptr;
                    }
                    if (g) cudaGraphDestroy(g);
                }
                (void)cudaGetLastError();
            }
            if (sgr.exec[0][lw]) {
                CPPHF_CUDA(cudaGraphLaunch(sgr.exec[0][lw], st));
                replayed = true;
            }
        }
        if (!replayed) CPPHF_TRY(body());
        pending_mix = false;
        int nslots = 0;
        int slots[kDiisMax];
        if (acc == 1) {
            // the history after this entry is added (oldest first), and the new
            // row of B: <R_slot, R_new> for each of its slots
            CPPHF_CUDA(cudaMemcpyAsync(Fh + (size_t)hhead * nel, F, fbytes, cudaMemcpyDeviceToDevice, st));
            const int m = std::min(hcount + 1, nh);
            for (int i = 0; i < m; ++i) slots[i] = ((hhead - (m - 1) + i) % nh + nh) % nh;
            nslots = m;
            FieldSet Hs;
            for (int i = 0; i < kDiisMax; ++i) Hs.p[i] = Rh + (size_t)slots[i < m ? i : 0] * nel;
            k_diis_dots<<<rgrid, 256, 0, st>>>(Hs, m, comm_out, K->w2d, nk, nb2, S, dots);
            CPPHF_LAUNCH_CHECK("diis dots");
            CPPHF_CUDA(cudaMemcpyAsync(dbuf, dots, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
        }
        // energy, grad_norm (density residual) and lam_pc (commutator residual) are
        // adjacent in DmScalars: one copy, plus mu
        static_assert(offsetof(DmScalars, lam_pc) == offsetof(DmScalars, energy) + 2 * sizeof(double),
                      "DmScalars read-back layout");
        CPPHF_CUDA(cudaMemcpyAsync(hbuf, &S->energy, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CPPHF_CUDA(cudaMemcpyAsync(hbuf + 3, mu_fin, sizeof(double), cudaMemcpyDeviceToHost, st));
        CPPHF_CUDA(cudaStreamSynchronize(st));
        if (!std::isfinite(hbuf[3]))
            return fail(CPPHF_ERR_TIMEOUT, "solve_scf: chemical-potential solve failed (device wait timeout or non-finite)");
        const double E_it = hbuf[0];
        const double d_res = std::sqrt(hbuf[1] / wsum);
        const double c_res = std::sqrt(hbuf[2] / wsum);
        converged = (d_res <= cfg->density_tol) && (c_res <= cfg->comm_tol);
        if (low && (converged || std::max(d_res, c_res) < cfg->mixed_switch_tol)) {
            // switch: mix as usual; the next build runs in complex128
            low = false;
            converged = false;
        }
        if (Dpre && !converged) CPPHF_CUDA(cudaMemcpyAsync(Dpre, D, fbytes, cudaMemcpyDeviceToDevice, st));
        d_hermitian = true;
        if (converged) {
            CPPHF_CUDA(cudaMemcpyAsync(D, Pn, fbytes, cudaMemcpyDeviceToDevice, st));
        } else if (acc == 1) {
            // ---- C-DIIS (solver_scf.hpp:253-349) ----
            const int m = nslots;
            const int newest = slots[m - 1];
            for (int i = 0; i < m; ++i) {
                Bs[(size_t)slots[i] * kDiisMax + newest] = dbuf[i];
                Bs[(size_t)newest * kDiisMax + slots[i]] = dbuf[i];
            }
            hcount = m;
            hhead = (hhead + 1) % nh;
            bool diis_ok = false;
            std::vector<double> sol;
            if (m >= std::max(2, (int)cfg->diis_start)) {
                const int n = m + 1;
                std::vector<double> A((size_t)n * n, 0.0);
                for (int i = 0; i < m; ++i) {
                    for (int j = 0; j < m; ++j) A[(size_t)i * n + j] = Bs[(size_t)slots[i] * kDiisMax + slots[j]];
                    A[(size_t)i * n + m] = -1.0;
                    A[(size_t)m * n + i] = -1.0;
                }
                diis_ok = diis_solve(A, n, sol);
            }
            if (diis_ok) {
                FieldSet Fs;
                DiisCoef cf;
                for (int i = 0; i < kDiisMax; ++i) {
                    Fs.p[i] = Fh + (size_t)slots[i < m ? i : 0] * nel;
                    cf.c[i] = i < m ? sol[(size_t)i] : 0.0;
                }
                const double damp = std::min(std::max(cfg->diis_damping, 0.0), 1.0);
                k_diis_extrapolate<<<egrid, 256, 0, st>>>(Fs, cf, m, damp, F, Fex, nel);
                CPPHF_LAUNCH_CHECK("diis extrapolate");
                CPPHF_TRY(hermitize(Fex, Fex, nk, nb, st));
                CPPHF_TRY(occupy(Fex, D));
            } else {
                CPPHF_TRY(mix_into_D(D, Pn, cfg->mixing));
            }
        } else if (acc == 2) {
            // ---- ODA (solver_scf.hpp:350-392): E(lambda) quadratic, one extra build ----
            CPPHF_TRY(build_fock(low ? &K32 : K, Pn, solver_sigma(low ? &K32 : K, Sn), Fn, nullptr, &mu2[2], nullptr, fws, L.fock_bytes, st));
            k_oda_c1<<<rgrid, 256, 0, st>>>(F, D, Pn, K->w2d, nk, nb, S, &mu2[3]);
            CPPHF_LAUNCH_CHECK("oda slope");
            double* const e2 = hbuf + 8 + kDiisMax;
            CPPHF_CUDA(cudaMemcpyAsync(e2, &mu2[2], 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
            CPPHF_CUDA(cudaStreamSynchronize(st));
            const double c1 = e2[1];
            const double c2 = (e2[0] - E_it) - c1;
            double lam;
            if (c2 > 1.0e-12)
                lam = std::min(std::max(-c1 / (2.0 * c2), 0.0), 1.0);
            else if (c1 < 0.0)
                lam = 1.0;
            else
                lam = 0.0;
            CPPHF_TRY(mix_into_D(D, Pn, lam));
        } else if (scf_graphs) {
            // the next iteration (or the finalisation) mixes first, unless the
            // residual pass has mixed D already
            if (!fuse_mix) pending_mix = true;
        } else {
            CPPHF_TRY(mix_into_D(D, Pn, cfg->mixing));
        }
        if (Dpre && !converged) {
            // ---- trust-radius clip (solver_scf.hpp:410-428) ----
            k_wdiff2<<<rgrid, 256, 0, st>>>(D, Dpre, K->w2d, nk, nb2, S, &mu2[2]);
            CPPHF_LAUNCH_CHECK("trust step norm");
            double* const hs2 = hbuf + 8 + kDiisMax + 2;
            CPPHF_CUDA(cudaMemcpyAsync(hs2, &mu2[2], sizeof(double), cudaMemcpyDeviceToHost, st));
            CPPHF_CUDA(cudaStreamSynchronize(st));
            const double s2 = *hs2;
            const double step = std::sqrt(s2 / wsum);
            if (step > cfg->trust_radius) CPPHF_TRY(mix_into_D(Dpre, D, cfg->trust_radius / step));
        }
        if (hist_E) hist_E[k] = E_it;
        if (hist_D) hist_D[k] = d_res;
        if (hist_C) hist_C[k] = c_res;
        ++k;
    }
    if (pending_mix) CPPHF_TRY(mix_into_D(D, Pn, cfg->mixing));
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

// Status of a synchronising entry point: a set device error word (a bounded
// wait that gave up during the call) wins over the call's own status.
int with_wait_check(int status, cudaStream_t st, const char* where) {
    const int w = check_wait_error(st, where);
    if (w == CPPHF_ERR_TIMEOUT || status == CPPHF_OK) return w;
    return status;
}

}  // namespace cpphf

extern "C" {

size_t cpphf_density_from_fock_workspace_bytes(int64_t nk, int64_t nb) {
    return cpphf::density_from_fock_workspace_bytes(nk, nb);
}

int cpphf_density_from_fock(const void* F, const double* w, int64_t nk1, int64_t nk2, int64_t nb, double n_e,
                            double T, double level_shift, void* P, double* eps, void* V, double* mu, void* workspace,
                            size_t workspace_bytes, void* stream) {
    const int s = cpphf::density_from_fock(static_cast<const double2*>(F), w, nk1, nk2, nb, n_e, T, level_shift,
                                           static_cast<double2*>(P), eps, static_cast<double2*>(V), mu, workspace,
                                           workspace_bytes, static_cast<cudaStream_t>(stream));
    return cpphf::with_wait_check(s, static_cast<cudaStream_t>(stream), "density_from_fock");
}

size_t cpphf_solve_dm_workspace_bytes(const cpphf_kernel* K) { return K ? cpphf::solve_dm_workspace_bytes(K) : 0; }

size_t cpphf_solve_dm_workspace_bytes_cfg(const cpphf_kernel* K, const cpphf_dm_config* cfg) {
    if (!K) return 0;
    if (cfg && cfg->optimizer == 1) return cpphf::solve_rtr_workspace_bytes(K, cfg);
    return cpphf::solve_dm_workspace_bytes(K);
}

int cpphf_solve_dm(const cpphf_kernel* K, const cpphf_dm_config* cfg, const void* P0, double n_e,
                   cpphf_project_fn project, void* project_user, void* Q_out, double* p_out, void* density_out,
                   void* fock_out, double* hist_E, double* hist_grad, cpphf_dm_result* result, void* workspace,
                   size_t workspace_bytes, void* stream) {
    const int s = cpphf::solve_dm(K, cfg, static_cast<const double2*>(P0), n_e, project, project_user,
                                  static_cast<double2*>(Q_out), p_out, static_cast<double2*>(density_out),
                                  static_cast<double2*>(fock_out), hist_E, hist_grad, result, workspace,
                                  workspace_bytes, static_cast<cudaStream_t>(stream));
    return cpphf::with_wait_check(s, static_cast<cudaStream_t>(stream), "solve_dm");
}

size_t cpphf_solve_scf_workspace_bytes(const cpphf_kernel* K) { return K ? cpphf::solve_scf_workspace_bytes(K) : 0; }

size_t cpphf_solve_scf_workspace_bytes_cfg(const cpphf_kernel* K, const cpphf_scf_config* cfg) {
    return K ? cpphf::solve_scf_workspace_bytes_cfg(K, cfg) : 0;
}

int cpphf_solve_scf(const cpphf_kernel* K, const cpphf_scf_config* cfg, const void* P0, double n_e,
                    cpphf_project_fn project, void* project_user, void* density_out, void* fock_out,
                    double* hist_E, double* hist_density, double* hist_comm, cpphf_scf_result* result,
                    void* workspace, size_t workspace_bytes, void* stream) {
    const int s = cpphf::solve_scf(K, cfg, static_cast<const double2*>(P0), n_e, project, project_user,
                                   static_cast<double2*>(density_out), static_cast<double2*>(fock_out), hist_E,
                                   hist_density, hist_comm, result, workspace, workspace_bytes,
                                   static_cast<cudaStream_t>(stream));
    return cpphf::with_wait_check(s, static_cast<cudaStream_t>(stream), "solve_scf");
}

}  // extern "C"
