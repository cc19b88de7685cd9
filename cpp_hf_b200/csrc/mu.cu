// Chemical-potential solvers as one cooperative persistent kernel each
// (cpp_hf utils.hpp:49-116).
//
// Every block owns a contiguous slice of the (nk*nb) eigenvalues.  Per round
// a block reduces its slice (fixed tree) into partials, the grid meets at a
// bounded barrier, every block sums all blocks' partials with the same fixed
// tree and replays the reference's scalar update rule itself, so the whole grid
// agrees on (lo, hi, mu).  The results are those of the reference's fixed
// iteration counts (30 bisection steps by default, mu_maxiter Newton steps).
// Bisection runs its first levels as exact multisection rounds, then finds
// the root of N(mu) = n_e by Newton and replays the remaining levels against
// it (a level whose midpoint lies within the rounding margin of the root is
// counted exactly), which reproduces the bisection's decisions with a few
// counts instead of one per level.  Newton stops early only once its state
// (mu, lo, hi) repeats with period 1 or 2, when the state after the remaining
// iterations is already known.
#include "common.cuh"
#include "mu.cuh"

#include <cstdlib>
#include <mutex>

namespace cpphf {

namespace {

constexpr int kMuThreads = 1024;
constexpr int kMuMaxGrid = 1024;
constexpr int kMuCache = 2;                           // eigenvalues a thread keeps in registers across rounds
constexpr int64_t kMuOneBlockMax = 32768;             // eigenvalues handled by a single CTA
constexpr int kMuCluster = 8;                         // CTAs of the cluster form (portable cluster size)
// eigenvalues handled by one cluster: up to 8 per thread and round; beyond
// that the cooperative grid's extra SMs outweigh its software barriers
constexpr int64_t kMuClusterMax = (int64_t)1 << 16;
constexpr int kBisectLevels = 3;                      // bisection steps per grid barrier
constexpr int kMuNV = (1 << kBisectLevels) - 1;       // midpoints evaluated per barrier
constexpr double kMuWide = 64.0;                      // exact multisection while the bracket exceeds 64 T
constexpr int kMuWarmMaxIter = 8;                     // Newton rounds from a warm start before the cold path
constexpr int kMuRootMaxIter = 80;                    // safeguarded Newton rounds (bisection fallback)

__device__ __forceinline__ double expit(double x) {
    if (x >= 0.0) return 1.0 / (1.0 + exp(-x));
    const double e = exp(x);
    return e / (1.0 + e);
}

// Shortcut thresholds on the (approximate) logistic argument x: for x >= 37,
// 1 + exp(-x) rounds to 1 in FP64, so expit(x) is exactly 1; for x <= -50,
// expit(x) < 2e-22 and the term is dropped (far below the rounding of any sum
// of weights it enters).  The approximate argument (difference times the
// reciprocal temperature) is within a few ulp of the exact quotient, far from
// either threshold's margin.
constexpr double kFdOne = 37.0;
constexpr double kFdZero = -50.0;

struct MuArgs {
    const double* eps;
    const double* w;  // per-k weights
    int64_t n;        // nk * nb
    int nb;
    double target;
    const double* mu0;  // device warm start (in-loop Newton; optional for the bisection's root) or null
    double T;
    int maxiter;
    int mode;  // 0 bisection (utils.hpp:49-75), 1 in-loop newton (utils.hpp:79-116)
    double* mu_out;
    double* part;     // [grid][2] min/max, then two [grid][kMuNV] partials buffers (by round parity)
    unsigned* sync;   // [0] count [1] gen [2] error
    unsigned* err;    // device error word (may be null)
    long long spin_limit;  // grid-barrier poll limit
};

// Element i of a block's slice in band-major order (band = i / nk, k = i % nk):
// the 32 lanes of a warp then hold one band at 32 neighbouring k-points, whose
// eigenvalues mostly fall on the same side of a trial mu, so the shortcut
// branches above stay warp-uniform.  eps is (nk, nb) row-major, w per k.
__device__ __forceinline__ void band_major(const MuArgs& a, unsigned i, unsigned nb, double& wk, double& e) {
    const unsigned nk = (unsigned)(a.n / nb);
    const unsigned band = i / nk, k = i - band * nk;
    wk = a.w[k];
    e = a.eps[(size_t)k * nb + band];
}

// Cluster barrier: every thread of every CTA of the cluster (hardware barrier;
// release / acquire at cluster scope orders the partials' global stores).
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Grid-wide synchronisation of the mu kernel.  CLUSTER = false: a cooperative
// grid with the bounded software barrier; CLUSTER = true: one thread-block
// cluster (kMuCluster CTAs) with the hardware cluster barrier.  In both, every
// block sums all blocks' partials itself in the same fixed order after the
// barrier (a few KB from L2; no block waits for a last arriver's reduction), so
// the partials are double-buffered by round parity (a block may start writing
// round r + 1 while another still reads round r).
template <bool CLUSTER>
struct MuSync {
    GridBarrier bar;
    double* ctot;  // shared totals
    double (*red)[32 * kMuNV];  // the kernel's block_sum scratch
    __device__ void init(const MuArgs& a, double* sh, double (*scratch)[32 * kMuNV]) {
        if (!CLUSTER) bar.init(a.sync, a.spin_limit, a.err);
        ctot = sh;
        red = scratch;
    }
    __device__ bool all() {
        if constexpr (CLUSTER) {
            cluster_sync_all();
            return true;
        } else {
            return bar.wait();
        }
    }
    // the partials buffer of a round
    __device__ double* partials(double* part, int round) const {
        return part + (size_t)(round & 1) * kMuNV * gridDim.x;
    }
    // every block's NV partials summed (fixed order); null if a wait gave up
    template <int NV>
    __device__ const double* reduce(const double* part, int G) {
        if constexpr (CLUSTER) {
            cluster_sync_all();
        } else {
            if (!bar.wait()) return nullptr;
        }
        // all threads load the partials at once (one L2 round trip), then the
        // block's fixed tree: every block forms the same totals
        double v[NV];
#pragma unroll
        for (int j = 0; j < NV; ++j) v[j] = 0.0;
        for (int b = threadIdx.x; b < G; b += blockDim.x) {
#pragma unroll
            for (int j = 0; j < NV; ++j) v[j] += __ldcg(&part[NV * b + j]);
        }
        block_sum<NV>(v, *red);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int j = 0; j < NV; ++j) ctot[j] = v[j];
        }
        __syncthreads();
        return ctot;
    }
    __device__ double load(const double* t, int j) const { return t[j]; }
};

template <bool CLUSTER>
__global__ void __launch_bounds__(kMuThreads) k_mu(MuArgs a) {
    __shared__ double red[32 * kMuNV];  // block_sum<kMuNV> scratch (32 doubles per value)
    __shared__ double ctot_sh[kMuNV];
    MuSync<CLUSTER> bar;
    bar.init(a, ctot_sh, &red);
    const int G = gridDim.x;
    const unsigned nb = (unsigned)a.nb;
    const unsigned n = (unsigned)a.n;
    const unsigned per = (n + G - 1) / G;  // (k, band) elements per block
    const unsigned e0 = blockIdx.x * per;
    const unsigned e1 = min(n, e0 + per);
    // The thread's eigenvalues and weights (band-major), loaded once: with at
    // most kMuCache of them per thread (the cooperative grid at the sizes the
    // solvers run) they stay in registers for every round; otherwise every
    // round reloads them.  Same elements, same order either way.
    const bool cached = (per + blockDim.x - 1) / blockDim.x <= (unsigned)kMuCache;  // grid-uniform
    double cw[kMuCache], ce[kMuCache];
#pragma unroll
    for (int u = 0; u < kMuCache; ++u) {
        const unsigned i = e0 + threadIdx.x + u * blockDim.x;
        cw[u] = 0.0;
        ce[u] = 0.0;
        if (cached && i < e1) band_major(a, i, nb, cw[u], ce[u]);
    }
    auto for_each_elem = [&](auto&& f) {
        if (cached) {
#pragma unroll
            for (int u = 0; u < kMuCache; ++u)
                if (e0 + threadIdx.x + u * blockDim.x < e1) f(cw[u], ce[u]);
        } else {
            for (unsigned i = e0 + threadIdx.x; i < e1; i += blockDim.x) {
                double wk, e;
                band_major(a, i, nb, wk, e);
                f(wk, e);
            }
        }
    };

    // 1. global min / max of eps
    double lmin = INFINITY, lmax = -INFINITY;
    for (unsigned i = e0 + threadIdx.x; i < e1; i += blockDim.x) {
        const double e = a.eps[i];
        lmin = fmin(lmin, e);
        lmax = fmax(lmax, e);
    }
    {
        double v[2] = {-lmin, lmax};
        // max-reduce through the sum scratch: use warp max then smem
        v[0] = warp_max(v[0]);
        v[1] = warp_max(v[1]);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0) {
            red[wid] = v[0];
            red[32 + wid] = v[1];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double m0 = -INFINITY, m1 = -INFINITY;
            for (int i = 0; i < nw; ++i) {
                m0 = fmax(m0, red[i]);
                m1 = fmax(m1, red[32 + i]);
            }
            a.part[2 * blockIdx.x] = m0;
            a.part[2 * blockIdx.x + 1] = m1;
        }
    }
    if (!bar.all()) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *a.mu_out = NAN;
        return;
    }
    // warp 0 reduces the block partials (fixed lane-strided order) and broadcasts
    __shared__ double bc[2];
    if (threadIdx.x < 32) {
        double m0 = -INFINITY, m1 = -INFINITY;
        for (int b = threadIdx.x; b < G; b += 32) {
            m0 = fmax(m0, __ldcg(&a.part[2 * b]));
            m1 = fmax(m1, __ldcg(&a.part[2 * b + 1]));
        }
        m0 = warp_max(m0);
        m1 = warp_max(m1);
        if (threadIdx.x == 0) {
            bc[0] = -m0;
            bc[1] = m1;
        }
    }
    __syncthreads();
    const double emin = bc[0], emax = bc[1];
    const double Tj = fmax(a.T, 1.0e-12);
    double lo, hi, mu = 0.0;
    if (a.mode == 0) {
        const double span = emax - emin + 10.0 * fmax(Tj, 1.0e-6);
        lo = emin - span;
        hi = emax + span;
    } else {
        lo = emin - 50.0 * Tj;
        hi = emax + 50.0 * Tj;
        mu = fmin(fmax(*a.mu0, lo), hi);
    }
    const double Tfd = Tj + 1.0e-12;  // fermidirac_scalar(x, Tj) = expit(-x / (Tj + 1e-12))
    const double invTfd = 1.0 / Tfd, invTj = 1.0 / Tj;
    double* part0 = a.part + 2 * G;  // two [G][kMuNV] partials buffers, by round parity
    __shared__ double bc_tot[kMuNV];
    int round = 0;
    if (a.mode == 0) {
        // Bisection (utils.hpp:49-75) in three phases.
        //  1. Exact multisection rounds while the bracket is wide: the counts at
        //     all midpoints of the next kBisectLevels levels of the bisection
        //     tree in one pass, then the tree is walked exactly as the
        //     sequential steps would.
        //  2. The root mu* of N(mu) = target by bracketed Newton from there.
        //  3. The remaining levels replayed against mu*: a midpoint farther than
        //     thr from mu* is decided by comparison (N is increasing, and there
        //     |N(mid) - target| >= 7 eps_N), a nearer one by its exact count.  A
        //     root with thr > T/8 (flat N, e.g. mu in a gap) runs the remaining
        //     levels as exact multisection rounds instead.
        const double epsN = 1.0e-13 * fmax(1.0, fabs(a.target));
        int it = 0;
        double Nlo = NAN, Nhi = NAN;  // counts at the bracket ends when evaluated
        bool ok = true;
        auto msec_round = [&]() {
            const int L = min(kBisectLevels, a.maxiter - it);
            const int nodes = (1 << L) - 1;
            double nlo[kMuNV], nhi[kMuNV], mid[kMuNV];
            nlo[0] = lo;
            nhi[0] = hi;
#pragma unroll
            for (int j = 0; j < kMuNV; ++j) {
                if (j < nodes) {
                    mid[j] = 0.5 * (nlo[j] + nhi[j]);
                    const int l = 2 * j + 1, r = 2 * j + 2;
                    if (l < kMuNV) {
                        nlo[l] = nlo[j];
                        nhi[l] = mid[j];
                    }
                    if (r < kMuNV) {
                        nlo[r] = mid[j];
                        nhi[r] = nhi[j];
                    }
                } else {
                    mid[j] = 0.0;
                }
            }
            double v[kMuNV];
#pragma unroll
            for (int j = 0; j < kMuNV; ++j) v[j] = 0.0;
            for_each_elem([&](double wk, double e) {
#pragma unroll
                for (int j = 0; j < kMuNV; ++j) {
                    if (j < nodes) {
                        // x = (mid - e) / Tfd: the term is exactly wk for x >= 37
                        // and below 2e-22 wk (dropped) for x <= -50
                        const double xa = (mid[j] - e) * invTfd;
                        if (xa >= kFdOne)
                            v[j] += wk;
                        else if (xa > kFdZero)
                            v[j] += wk * expit(-(e - mid[j]) / Tfd);
                    }
                }
            });
            block_sum<kMuNV>(v, red);
            double* part = bar.partials(part0, round);
            if (threadIdx.x == 0) {
#pragma unroll
                for (int j = 0; j < kMuNV; ++j) __stcg(&part[kMuNV * blockIdx.x + j], v[j]);
            }
            const double* tot = bar.template reduce<kMuNV>(part, G);
            if (!tot) {
                ok = false;
                return;
            }
            if (threadIdx.x < kMuNV) bc_tot[threadIdx.x] = bar.load(tot, threadIdx.x);
            __syncthreads();
            int node = 0;
            for (int l = 0; l < L; ++l) {
                double m = mid[0];
#pragma unroll
                for (int j = 1; j < kMuNV; ++j)
                    if (j == node) m = mid[j];
                if (bc_tot[node] > a.target) {
                    hi = m;
                    Nhi = bc_tot[node];
                    node = 2 * node + 1;
                } else {
                    lo = m;
                    Nlo = bc_tot[node];
                    node = 2 * node + 2;
                }
            }
            __syncthreads();
            it += L;
            ++round;
        };
        // count N and slope Z = dN/dmu at one mu (one grid round)
        auto count_round = [&](double m, double& N, double& Z) {
            double v[2] = {0.0, 0.0};
            for_each_elem([&](double wk, double e) {
                const double xa = (m - e) * invTfd;
                if (xa >= kFdOne) {
                    v[0] += wk;
                } else if (xa > kFdZero) {
                    const double pf = expit(-(e - m) / Tfd);
                    v[0] += wk * pf;
                    v[1] += wk * pf * (1.0 - pf) * invTfd;
                }
            });
            block_sum<2>(v, red);
            double* part = bar.partials(part0, round);
            if (threadIdx.x == 0) {
                __stcg(&part[2 * blockIdx.x], v[0]);
                __stcg(&part[2 * blockIdx.x + 1], v[1]);
            }
            const double* tot = bar.template reduce<2>(part, G);
            ++round;
            if (!tot) {
                ok = false;
                return;
            }
            if (threadIdx.x < 2) bc_tot[threadIdx.x] = bar.load(tot, threadIdx.x);
            __syncthreads();
            N = bc_tot[0];
            Z = bc_tot[1];
            __syncthreads();
        };
        // safeguarded Newton for the root of N(mu) = target inside [ra, rb]
        struct Root {
            double m, g, slope;
            bool conv;
        };
        auto newton = [&](double m, double ra, double rb, int maxit) {
            Root R{m, INFINITY, 0.0, false};
            for (int r = 0; ok && r < maxit; ++r) {
                double N = 0.0, Z = 0.0;
                count_round(R.m, N, Z);
                if (!ok) break;
                R.g = N - a.target;
                R.slope = Z;
                if (fabs(R.g) <= epsN) {
                    R.conv = true;
                    break;
                }
                if (R.g > 0.0)
                    rb = R.m;
                else
                    ra = R.m;
                double mn = (Z > 0.0) ? R.m - R.g / Z : NAN;
                if (!(mn > ra && mn < rb)) mn = 0.5 * (ra + rb);
                if (mn == R.m) break;
                R.m = mn;
            }
            return R;
        };
        // replay the levels left against the root when its threshold allows
        auto replay = [&](const Root& R) {
            const double thr = (R.conv && R.slope > 0.0) ? 8.0 * (fabs(R.g) + epsN) / R.slope : INFINITY;
            if (!(ok && thr <= 0.125 * Tj)) return false;
            for (; ok && it < a.maxiter; ++it) {
                const double md = 0.5 * (lo + hi);
                bool up;
                if (fabs(md - R.m) > thr) {
                    up = md > R.m;
                } else {
                    double N = 0.0, Z = 0.0;
                    count_round(md, N, Z);
                    up = N > a.target;
                }
                if (up)
                    hi = md;
                else
                    lo = md;
            }
            return true;
        };
        // A warm start (the caller's previous mu, e.g. the last SCF iteration's)
        // inside the initial bracket: Newton from there over the whole bracket and,
        // if it converges, every level replayed from the top.  The levels depend
        // only on the root, so the result is the same as from a cold start.
        bool done = false;
        if (a.mu0 && a.maxiter > 0) {
            const double warm = *a.mu0;
            if (isfinite(warm) && warm > lo && warm < hi) {
                const Root R = newton(warm, lo, hi, kMuWarmMaxIter);
                done = ok && replay(R);
            }
        }
        if (!done && ok) {
            while (ok && it < a.maxiter && (it == 0 || hi - lo > kMuWide * Tj)) msec_round();
            if (ok && it < a.maxiter) {
                // 2. root: secant start inside the bracket, then safeguarded Newton
                double m = 0.5 * (lo + hi);
                if (isfinite(Nlo) && isfinite(Nhi) && Nhi > Nlo) {
                    const double ms = lo + (a.target - Nlo) * (hi - lo) / (Nhi - Nlo);
                    if (ms > lo && ms < hi) m = ms;
                }
                const Root R = newton(m, lo, hi, kMuRootMaxIter);
                // 3. replay, or exact multisection for a flat N
                if (!replay(R))
                    while (ok && it < a.maxiter) msec_round();
            }
        }
        if (!ok) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *a.mu_out = NAN;
            return;
        }
    } else {
        // Newton in a bracket.  The update is a deterministic function of the
        // state (mu, lo, hi); once the state repeats with period 1 or 2 the
        // remaining iterations are known, so the loop stops there with the state
        // the full iteration count would end in.
        double mu1 = NAN, lo1 = NAN, hi1 = NAN;  // state one iteration back
        for (int it = 0; it < a.maxiter; ++it) {
            double v[2] = {0.0, 0.0};
            for_each_elem([&](double wk, double e) {
                // p = expit((mu - e) / Tj) is exactly 1 (and p (1 - p) exactly 0)
                // for an argument >= 37; below -50 both terms are dropped
                const double xa = (mu - e) * invTj;
                if (xa >= kFdOne) {
                    v[0] += wk;
                } else if (xa > kFdZero) {
                    const double p = expit((mu - e) / Tj);
                    v[0] += wk * p;
                    v[1] += wk * p * (1.0 - p) / Tj;
                }
            });
            block_sum<2>(v, red);
            double* part = bar.partials(part0, it);
            if (threadIdx.x == 0) {
                __stcg(&part[2 * blockIdx.x], v[0]);
                __stcg(&part[2 * blockIdx.x + 1], v[1]);
            }
            const double* tot = bar.template reduce<2>(part, G);
            if (!tot) {
                if (blockIdx.x == 0 && threadIdx.x == 0) *a.mu_out = NAN;
                return;
            }
            if (threadIdx.x < 2) bc_tot[threadIdx.x] = bar.load(tot, threadIdx.x);
            __syncthreads();
            const double N = bc_tot[0], Z = bc_tot[1];
            __syncthreads();
            const double mu0 = mu, lo0 = lo, hi0 = hi;
            const double g = N - a.target;
            if (g < 0.0) lo = mu;
            if (g > 0.0) hi = mu;
            const double Zs = fmax(Z, 1.0e-18);
            double mn = mu - g / Zs;
            const double mb = 0.5 * (lo + hi);
            if (mn <= lo || mn >= hi) mn = mb;
            mn = fmin(fmax(mn, lo), hi);
            if (!isfinite(mn)) mn = mb;
            mu = mn;
            const int rest = a.maxiter - (it + 1);
            if (mu == mu0 && lo == lo0 && hi == hi0) break;  // fixed point
            if (mu == mu1 && lo == lo1 && hi == hi1) {       // period 2: (s1, s0) repeats
                if (rest & 1) mu = mu0;
                break;
            }
            mu1 = mu0;
            lo1 = lo0;
            hi1 = hi0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.mu_out = (a.mode == 0) ? 0.5 * (lo + hi) : mu;
}

// Largest cooperative grid: the resident blocks of the device, at most kMuMaxGrid.
int max_coop_grid() {
    static int g = 0;
    static std::once_flag once;
    std::call_once(once, [] {
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_mu<false>, kMuThreads, 0);
        if (per < 1) per = 1;
        g = std::min(kMuMaxGrid, per * num_sms());
    });
    return g;
}


// ---------------------------------------------------------------------------
// Allocation-free bisection entry point.  Its scratch (grid-barrier words and
// block partials, the same layout the workspace variant uses) is this
// file-scope array, sized for the largest cooperative grid the solver ever
// launches.  Every GPU that loads the library holds it until the process
// exits; every call shares it.
// ---------------------------------------------------------------------------
constexpr size_t kMuNoAllocScratchBytes = 64 + sizeof(double) * ((2 + 2 * kMuNV) * (size_t)kMuMaxGrid + 2 * kMuNV);
static __device__ __align__(256) unsigned char g_mu_noalloc_scratch[kMuNoAllocScratchBytes];

}  // namespace

size_t mu_workspace_bytes(int64_t, int64_t) {
    return 64 + sizeof(double) * ((2 + 2 * kMuNV) * (size_t)kMuMaxGrid + 2 * kMuNV);
}

int mu_solve(const double* eps, const double* w, int64_t nk, int64_t nb, double target,
             const double* mu0, double T, int maxiter, int mode, double* mu_out, void* ws,
             size_t wsb, cudaStream_t st) {
    if (nk < 1 || nb < 1) return fail(CPPHF_ERR_INVALID, "mu: empty eigenvalue array");
    if (nb > (((int64_t)1 << 31) - 1) / nk) return fail(CPPHF_ERR_INVALID, "mu: more than 2^31-1 eigenvalues");
    if (!eps || !w || !mu_out) return fail(CPPHF_ERR_INVALID, "mu: null pointer");
    if (mode == 1 && !mu0) return fail(CPPHF_ERR_INVALID, "mu: null warm start");
    if (!ws || wsb < mu_workspace_bytes(nk, nb)) return fail(CPPHF_ERR_INVALID, "mu: workspace too small");
    const int64_t n = nk * nb;
    int grid = (int)std::min<int64_t>(max_coop_grid(), (n + kMuThreads - 1) / kMuThreads);
    if (grid < 1) grid = 1;
    // small problems: one CTA does it all (its barriers are block-local), launched
    // as an ordinary kernel so that solves on other streams keep running beside it
    if (n <= kMuOneBlockMax) grid = 1;
    MuArgs a;
    a.eps = eps;
    a.w = w;
    a.n = n;
    a.nb = (int)nb;
    a.target = target;
    a.mu0 = mu0;
    a.T = T;
    a.maxiter = maxiter;
    a.mode = mode;
    a.mu_out = mu_out;
    a.sync = reinterpret_cast<unsigned*>(ws);
    a.err = wait_error_word();
    if (!a.err) return CPPHF_ERR_CUDA;
    a.spin_limit = barrier_spin_limit();
    a.part = reinterpret_cast<double*>(static_cast<unsigned char*>(ws) + 64);
    CPPHF_CUDA(cudaMemsetAsync(ws, 0, 64, st));
    if (grid == 1) {
        k_mu<false><<<1, kMuThreads, 0, st>>>(a);
        CPPHF_LAUNCH_CHECK("mu (one block)");
        return CPPHF_OK;
    }
    if (n <= kMuClusterMax) {
        // mid-size problems: one cluster of kMuCluster CTAs, hardware cluster
        // barriers between the rounds (no software grid barrier)
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kMuCluster);
        cfg.blockDim = dim3(kMuThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kMuCluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CPPHF_CUDA(cudaLaunchKernelEx(&cfg, k_mu<true>, a));
        return CPPHF_OK;
    }
    void* args[] = {&a};
    CPPHF_CUDA(cudaLaunchCooperativeKernel((const void*)k_mu<false>, dim3(grid), dim3(kMuThreads), args, 0, st));
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

size_t cpphf_mu_workspace_bytes(int64_t nk, int64_t nb) { return cpphf::mu_workspace_bytes(nk, nb); }

int cpphf_find_mu_bisection(const double* eps, const double* weights, int64_t nk, int64_t nb,
                            double n_e, double T, int maxiter, double* mu_out, void* workspace,
                            size_t workspace_bytes, void* stream) {
    if (maxiter <= 0) maxiter = 30;
    return cpphf::mu_solve(eps, weights, nk, nb, n_e, nullptr, T, maxiter, 0, mu_out, workspace,
                           workspace_bytes, static_cast<cudaStream_t>(stream));
}

// The device address of g_mu_noalloc_scratch for the current device.  Host
// code only sees a host-side stand-in for the array under that name, so the
// address is looked up once per device with that device current (first call on
// the device; keep that call outside stream capture) and cached.
static int noalloc_scratch(void** out) {
    static std::mutex mtx;
    static void* ptrs[64] = {nullptr};
    int dev = 0;
    CPPHF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cpphf::fail(CPPHF_ERR_UNSUPPORTED, "find_mu_bisection_noalloc: device index >= 64");
    std::lock_guard<std::mutex> lock(mtx);
    if (!ptrs[dev]) {
        void* p = nullptr;
        CPPHF_CUDA(cudaGetSymbolAddress(&p, cpphf::g_mu_noalloc_scratch));
        ptrs[dev] = p;
    }
    *out = ptrs[dev];
    return CPPHF_OK;
}

int cpphf_find_mu_bisection_noalloc(const double* eps, const double* weights, int64_t nk, int64_t nb, double n_e,
                                    double T, int maxiter, double* mu_out, void* stream) {
    if (nk < 1 || nb < 1) return cpphf::fail(CPPHF_ERR_INVALID, "mu: empty eigenvalue array");
    if (nb > CPPHF_MU_NOALLOC_MAX_EIGENVALUES / nk)
        return cpphf::fail(CPPHF_ERR_INVALID, "find_mu_bisection_noalloc: nk*nb exceeds the maximum of 2^31-1 eigenvalues");
    void* scratch = nullptr;
    CPPHF_TRY(noalloc_scratch(&scratch));
    if (maxiter <= 0) maxiter = 30;
    return cpphf::mu_solve(eps, weights, nk, nb, n_e, nullptr, T, maxiter, 0, mu_out, scratch,
                           cpphf::kMuNoAllocScratchBytes, static_cast<cudaStream_t>(stream));
}

int cpphf_solve_mu_inloop(const double* eps, const double* w_norm, int64_t nk, int64_t nb,
                          double n_target_norm, const double* mu0, double T, int maxiter,
                          double* mu_out, void* workspace, size_t workspace_bytes, void* stream) {
    return cpphf::mu_solve(eps, w_norm, nk, nb, n_target_norm, mu0, T, maxiter, 1, mu_out, workspace,
                           workspace_bytes, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
