// Batched Hermitian eigendecomposition by cyclic complex Jacobi sweeps
// (replaces Eigen's SelfAdjointEigenSolver in cpp_hf linalg.hpp:39-66).
//
// One team per matrix: a warp for nb <= 16 (several matrices per CTA), the
// whole CTA for larger nb.  The matrix and its accumulated eigenvectors live in
// shared memory (row stride nb+1 against bank conflicts).  Each sweep runs the
// nb-1 rounds of a round-robin (circle) ordering; a round rotates nb/2
// disjoint (p, q) pairs at once with
//     J = [[c, s e^{i phi}], [-s e^{-i phi}, c]],  A_pq = |A_pq| e^{i phi},
// (c, s) the real symmetric Schur rotation of [[A_pp, |A_pq|], [|A_pq|, A_qq]],
// applied as A <- J^H A (rows), A <- A J and V <- V J (columns); the 2x2 pivot
// block is then written exactly (A_pp - t|A_pq|, A_qq + t|A_pq|, zeros).
// Sweeps stop when the off-diagonal Frobenius norm falls to nb * eps of the
// total (the rounding level of the rotations), when a sweep no longer reduces
// it, or after kMaxSweeps.  Eigenvalues are sorted ascending (stable),
// eigenvector columns permuted to match.
#include "common.cuh"
#include "eigh.cuh"

#include <cstring>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

namespace cpphf {

namespace {

constexpr int kMaxSweeps = 40;
constexpr int kWarpTeamMaxNb = 16;
constexpr int kWarpTeamsPerCta = 4;
constexpr int kCtaTeamThreads = 256;

struct PairParam {
    double c;
    double2 sig;
    double npp, nqq;
    int p, q;
};

template <bool WARP>
__device__ __forceinline__ void team_sync() {
    if (WARP)
        __syncwarp();
    else
        __syncthreads();
}

template <bool WARP>
__device__ __forceinline__ double team_sum(double v, double* red) {
    if (WARP) return warp_sum(v);
    double a[1] = {v};
    block_sum<1>(a, *reinterpret_cast<double(*)[32]>(red));  // red: the kernel's 32-double scratch
    return a[0];
}

__device__ __forceinline__ void pair_of(int r, int k, int m, int& p, int& q) {
    // circle method over m (even) players: m-1 fixed, others rotate
    if (k == 0) {
        p = r;
        q = m - 1;
    } else {
        p = (r + k) % (m - 1);
        q = (r - k + (m - 1)) % (m - 1);
    }
    if (p > q) {
        int t = p;
        p = q;
        q = t;
    }
}

// Jacobi on A (nb x nb, stride ld) accumulating V.  `tid`/`nt` index the team.
template <bool WARP>
__device__ void jacobi(double2* A, double2* V, int nb, int ld, PairParam* pp, double* red, int tid,
                       int nt) {
    for (int e = tid; e < nb * nb; e += nt) {
        const int i = e / nb, j = e - i * nb;
        V[i * ld + j] = mk(i == j ? 1.0 : 0.0, 0.0);
    }
    team_sync<WARP>();
    if (nb == 1) return;
    const int m = nb + (nb & 1);
    const int npair = m / 2;
    // converged once the off-diagonal norm is at the rounding level of the
    // rotations, (nb eps)^2 of the total (squared Frobenius norms), or once a
    // sweep no longer reduces it
    const double thr = (double)nb * 2.220446049250313e-16;
    double off_prev = INFINITY;
    for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int e = tid; e < nb * nb; e += nt) {
            const int i = e / nb, j = e - i * nb;
            const double2 a = A[i * ld + j];
            const double m2 = a.x * a.x + a.y * a.y;
            tot += m2;
            if (i != j) off += m2;
        }
        off = team_sum<WARP>(off, red);
        tot = team_sum<WARP>(tot, red);
        if (!(off > thr * thr * tot) || off == 0.0 || !(off < off_prev)) break;
        off_prev = off;
        for (int r = 0; r < m - 1; ++r) {
            for (int k = tid; k < npair; k += nt) {
                int p, q;
                pair_of(r, k, m, p, q);
                PairParam P;
                P.p = p;
                P.q = q;
                P.c = 1.0;
                P.sig = mk(0.0, 0.0);
                if (q < nb) {
                    const double app = A[p * ld + p].x, aqq = A[q * ld + q].x;
                    const double2 b = A[p * ld + q];
                    const double ab = hypot(b.x, b.y);
                    P.npp = app;
                    P.nqq = aqq;
                    if (ab > 0.0) {
                        const double tau = (aqq - app) / (2.0 * ab);
                        double t;
                        if (fabs(tau) > 1e150)
                            t = 0.5 / tau;
                        else
                            t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        const double c = 1.0 / sqrt(1.0 + t * t);
                        const double s = t * c;
                        P.c = c;
                        P.sig = mk(s * (b.x / ab), s * (b.y / ab));
                        P.npp = app - t * ab;
                        P.nqq = aqq + t * ab;
                    }
                } else {
                    P.q = -1;
                }
                pp[k] = P;
            }
            team_sync<WARP>();
            // rows: A <- J^H A
            for (int e = tid; e < npair * nb; e += nt) {
                const int k = e / nb, j = e - k * nb;
                const PairParam P = pp[k];
                if (P.q < 0 || (P.sig.x == 0.0 && P.sig.y == 0.0)) continue;
                const double2 ap = A[P.p * ld + j], aq = A[P.q * ld + j];
                double2 np_ = cscale(ap, P.c), nq = cscale(aq, P.c);
                np_ = csub(np_, cmul(P.sig, aq));
                nq = cadd(nq, cmul(cconj(P.sig), ap));
                A[P.p * ld + j] = np_;
                A[P.q * ld + j] = nq;
            }
            team_sync<WARP>();
            // columns: A <- A J, V <- V J; exact pivot block
            for (int e = tid; e < npair * nb; e += nt) {
                const int k = e / nb, i = e - k * nb;
                const PairParam P = pp[k];
                if (P.q < 0 || (P.sig.x == 0.0 && P.sig.y == 0.0)) continue;
                if (i == P.p) {
                    A[P.p * ld + P.p] = mk(P.npp, 0.0);
                    A[P.p * ld + P.q] = mk(0.0, 0.0);
                } else if (i == P.q) {
                    A[P.q * ld + P.p] = mk(0.0, 0.0);
                    A[P.q * ld + P.q] = mk(P.nqq, 0.0);
                } else {
                    const double2 ap = A[i * ld + P.p], aq = A[i * ld + P.q];
                    A[i * ld + P.p] = csub(cscale(ap, P.c), cmul(cconj(P.sig), aq));
                    A[i * ld + P.q] = cadd(cmul(P.sig, ap), cscale(aq, P.c));
                }
                const double2 vp = V[i * ld + P.p], vq = V[i * ld + P.q];
                V[i * ld + P.p] = csub(cscale(vp, P.c), cmul(cconj(P.sig), vq));
                V[i * ld + P.q] = cadd(cmul(P.sig, vp), cscale(vq, P.c));
            }
            team_sync<WARP>();
        }
    }
}

// Input transform: 0 -> herm(M), 1 -> herm(i M).
template <bool WARP>
__global__ void k_eigh(const double2* __restrict__ M, double* __restrict__ w, double2* __restrict__ Vout,
                       int64_t batch, int nb, int mode, BlockSpec bs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ld = nb + 1;
    const int teams = WARP ? (blockDim.x >> 5) : 1;
    const int team = WARP ? (threadIdx.x >> 5) : 0;
    const int tid = WARP ? (threadIdx.x & 31) : threadIdx.x;
    const int nt = WARP ? 32 : blockDim.x;
    const size_t mat = (size_t)nb * ld;
    const int npair = (nb + 1) / 2 + 1;
    unsigned char* base = smem_raw;
    double2* A = reinterpret_cast<double2*>(base) + (size_t)team * 2 * mat;
    double2* V = A + mat;
    base += sizeof(double2) * 2 * mat * teams;
    PairParam* pp = reinterpret_cast<PairParam*>(base) + (size_t)team * npair;
    base += sizeof(PairParam) * npair * teams;
    int* rank = reinterpret_cast<int*>(base) + (size_t)team * nb;
    base += sizeof(int) * nb * teams;
    double* red = reinterpret_cast<double*>(((uintptr_t)base + 7) & ~(uintptr_t)7);

    const int64_t k = (int64_t)blockIdx.x * teams + team;
    const bool active = k < batch;  // whole team shares k
    if (active) {
        const double2* Mk = M + (size_t)k * nb * nb;
        for (int e = tid; e < nb * nb; e += nt) {
            const int i = e / nb, j = e - i * nb;
            double2 a = Mk[i * nb + j], b = Mk[j * nb + i];
            if (mode == 1) {  // i*M
                a = mk(-a.y, a.x);
                b = mk(-b.y, b.x);
            }
            double2 h = mk(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
            if (i == j) h.y = 0.0;
            if (bs.nblocks > 1 && bs.blk[i] != bs.blk[j]) h = mk(0.0, 0.0);
            A[i * ld + j] = h;
        }
    }
    if (!WARP) __syncthreads();
    if (WARP && !active) return;  // warp-uniform
    if (!WARP && !active) return;  // block-uniform
    team_sync<WARP>();
    jacobi<WARP>(A, V, nb, ld, pp, red, tid, nt);
    // stable ascending ranks (within each block when bs.sort_within)
    for (int i = tid; i < nb; i += nt) {
        const double di = A[i * ld + i].x;
        int r = 0;
        if (bs.nblocks > 1 && !bs.sort) {
            const int bi = bs.blk[i];
            r = bs.start[bi];
            for (int j = bs.start[bi]; j < bs.start[bi + 1]; ++j) {
                const double dj = A[j * ld + j].x;
                if (dj < di || (dj == di && j < i)) ++r;
            }
        } else {
            for (int j = 0; j < nb; ++j) {
                const double dj = A[j * ld + j].x;
                if (dj < di || (dj == di && j < i)) ++r;
            }
        }
        rank[i] = r;
    }
    team_sync<WARP>();
    double* wk = w + (size_t)k * nb;
    double2* Vk = Vout + (size_t)k * nb * nb;
    for (int i = tid; i < nb; i += nt) wk[rank[i]] = A[i * ld + i].x;
    for (int e = tid; e < nb * nb; e += nt) {
        const int r = e / nb, c = e - r * nb;
        Vk[r * nb + rank[c]] = V[r * ld + c];
    }
}


// max |M_ij| over the off-block entries of every matrix (linalg.hpp:123-140).
__global__ void k_max_offblock(const double2* __restrict__ M, int64_t batch, int nb, BlockSpec bs,
                               unsigned long long* out) {
    const int64_t n = batch * (int64_t)nb * nb;
    double m = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % ((int64_t)nb * nb));
        const int i = r / nb, j = r - i * nb;
        if (bs.blk[i] != bs.blk[j]) {
            const double2 a = M[e];
            m = fmax(m, hypot(a.x, a.y));
        }
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// max |M| (out[0]) and max |M_ij| over the off-block entries (out[1]) of a
// batch, as doubles reinterpreted for atomicMax (non-negative, so the integer
// order is the numeric order).
__global__ void k_block_norms(const double2* __restrict__ M, int64_t batch, int nb, BlockSpec bs,
                              unsigned long long* out) {
    const int64_t n = batch * (int64_t)nb * nb;
    double all = 0.0, off = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % ((int64_t)nb * nb));
        const int i = r / nb, j = r - i * nb;
        const double2 a = M[e];
        const double v = hypot(a.x, a.y);
        all = fmax(all, v);
        if (bs.blk[i] != bs.blk[j]) off = fmax(off, v);
    }
    all = warp_max(all);
    off = warp_max(off);
    if ((threadIdx.x & 31) == 0) {
        if (all > 0.0) atomicMax(&out[0], (unsigned long long)__double_as_longlong(all));
        if (off > 0.0) atomicMax(&out[1], (unsigned long long)__double_as_longlong(off));
    }
}

size_t eigh_smem(int nb, bool warp) {
    const int teams = warp ? kWarpTeamsPerCta : 1;
    const size_t mat = (size_t)nb * (nb + 1);
    const int npair = (nb + 1) / 2 + 1;
    return (sizeof(double2) * 2 * mat + sizeof(PairParam) * npair + sizeof(int) * nb) * teams + 8 +
           sizeof(double) * 32;
}

}  // namespace

int eigh_batched(const double2* M, double* w, double2* V, int64_t batch, int64_t nb, int mode,
                 const BlockSpec* bs_in, cudaStream_t st) {
    if (nb < 1 || batch < 0) return fail(CPPHF_ERR_INVALID, "eigh: invalid shape");
    if (batch == 0) return CPPHF_OK;
    if (nb > kMaxEighNb)
        return fail(CPPHF_ERR_UNSUPPORTED, "eigh: nb > " + std::to_string(kMaxEighNb) + " not supported");
    BlockSpec bs;
    if (bs_in)
        bs = *bs_in;
    else {
        bs.nblocks = 1;
        bs.sort = 1;
        bs.start[0] = 0;
        bs.start[1] = (short)nb;
        for (int i = 0; i < nb; ++i) bs.blk[i] = 0;
    }
    if (bs.nblocks <= 1 && eigh_small_enabled(nb)) return eigh_small(M, w, V, batch, nb, mode, st);
    static std::once_flag once;
    std::call_once(once, [] {
        raise_smem(k_eigh<true>);
        raise_smem(k_eigh<false>);
    });
    if (nb <= kWarpTeamMaxNb) {
        const size_t smem = eigh_smem((int)nb, true);
        const int64_t grid = (batch + kWarpTeamsPerCta - 1) / kWarpTeamsPerCta;
        k_eigh<true><<<(unsigned)grid, 32 * kWarpTeamsPerCta, smem, st>>>(M, w, V, batch, (int)nb, mode, bs);
    } else {
        const size_t smem = eigh_smem((int)nb, false);
        k_eigh<false><<<(unsigned)batch, kCtaTeamThreads, smem, st>>>(M, w, V, batch, (int)nb, mode, bs);
    }
    CPPHF_LAUNCH_CHECK("eigh");
    return CPPHF_OK;
}

int block_structure_ok(const double2* M, int64_t batch, int64_t nb, const BlockSpec& bs, unsigned long long* dev2,
                       cudaStream_t st, bool* ok) {
    *ok = true;
    if (batch <= 0) return CPPHF_OK;
    CPPHF_CUDA(cudaMemsetAsync(dev2, 0, 2 * sizeof(unsigned long long), st));
    const int64_t n = batch * nb * nb;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8));
    k_block_norms<<<grid, 256, 0, st>>>(M, batch, (int)nb, bs, dev2);
    CPPHF_LAUNCH_CHECK("block structure check");
    unsigned long long h[2] = {0ull, 0ull};
    CPPHF_CUDA(cudaMemcpyAsync(h, dev2, sizeof(h), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    double scale, off;
    std::memcpy(&scale, &h[0], sizeof(double));
    std::memcpy(&off, &h[1], sizeof(double));
    *ok = off <= 1.0e-10 + 1.0e-10 * scale;
    return CPPHF_OK;
}

int make_block_spec(int64_t nb, const int64_t* sizes, int64_t n_sizes, int sort, BlockSpec& bs) {
    if (n_sizes < 1 || n_sizes > kMaxEighNb) return fail(CPPHF_ERR_INVALID, "block sizes must sum to nb");
    int64_t tot = 0;
    for (int64_t b = 0; b < n_sizes; ++b) {
        if (sizes[b] <= 0) return fail(CPPHF_ERR_INVALID, "block_sizes entries must be positive.");
        tot += sizes[b];
    }
    if (tot != nb) return fail(CPPHF_ERR_INVALID, "block sizes must sum to nb");
    bs.nblocks = (int)n_sizes;
    bs.sort = sort ? 1 : 0;
    int s0 = 0;
    for (int b = 0; b < n_sizes; ++b) {
        bs.start[b] = (short)s0;
        for (int i = 0; i < sizes[b]; ++i) bs.blk[s0 + i] = (unsigned char)b;
        s0 += (int)sizes[b];
    }
    bs.start[n_sizes] = (short)s0;
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

int cpphf_eigh_batched(const void* M, double* w, void* V, int64_t batch, int64_t nb, void* stream) {
    return cpphf::eigh_batched(static_cast<const double2*>(M), w, static_cast<double2*>(V), batch, nb,
                               0, nullptr, static_cast<cudaStream_t>(stream));
}

int cpphf_eigh_block_sizes(const void* M, double* w, void* V, int64_t batch, int64_t nb,
                           const int64_t* sizes, int64_t n_sizes, int sort, void* stream) {
    cpphf::BlockSpec bs;
    CPPHF_TRY(cpphf::make_block_spec(nb, sizes, n_sizes, sort, bs));
    return cpphf::eigh_batched(static_cast<const double2*>(M), w, static_cast<double2*>(V), batch, nb,
                               0, &bs, static_cast<cudaStream_t>(stream));
}


int cpphf_max_offblock_sizes(const void* M, int64_t batch, int64_t nb, const int64_t* sizes, int64_t n_sizes,
                             double* out, void* stream) {
    cpphf::BlockSpec bs;
    int64_t tot = 0;
    for (int64_t b = 0; b < n_sizes; ++b) tot += sizes[b];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CPPHF_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
    if (nb > cpphf::kMaxEighNb || n_sizes < 1 || tot != nb || batch <= 0) {
        // linalg.hpp:123-140 tolerates any sizes; only the covered region is masked
        if (nb > cpphf::kMaxEighNb) return cpphf::fail(CPPHF_ERR_UNSUPPORTED, "max_offblock_sizes: nb too large");
        if (batch <= 0) return CPPHF_OK;
    }
    bs.nblocks = 0;
    bs.sort = 1;
    // entries outside every listed block belong to their own pseudo-block
    for (int i = 0; i < nb; ++i) bs.blk[i] = (unsigned char)(100 + i);  // unique id per uncovered index
    int s0 = 0;
    for (int64_t b = 0; b < n_sizes && b < 100; ++b) {
        for (int64_t i = 0; i < sizes[b] && s0 + i < nb; ++i) bs.blk[s0 + i] = (unsigned char)b;
        s0 += (int)sizes[b];
    }
    const int64_t n = batch * nb * nb;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096));
    cpphf::k_max_offblock<<<grid, 256, 0, st>>>(static_cast<const double2*>(M), batch, (int)nb, bs,
                                                reinterpret_cast<unsigned long long*>(out));
    CPPHF_LAUNCH_CHECK("max_offblock");
    return CPPHF_OK;
}

int cpphf_cayley_spectral_setup(const void* d, void* V, double* lam, int64_t batch, int64_t nb,
                                void* stream) {
    return cpphf::eigh_batched(static_cast<const double2*>(d), lam, static_cast<double2*>(V), batch,
                               nb, 1, nullptr, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
