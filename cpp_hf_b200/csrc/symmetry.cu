// Symmetry-averaging projector on device fields (cpp_hf src/cpp_hf/symmetry.py:18-117),
// usable directly as a solver's projector (cpphf_project_fn) so that symmetric
// solves need no host round trip.
//
// Pass 1 (group average): out(k) = (sum_g g A(k) g^H + sum_s s A(-k) s^H) / N over the
// unitary group G (or the identity when only a spatial group is given) and the
// spatial group S (symmetry.py:44-75).  Pass 2 (time reversal): out(k) =
// (B(k) + U conj(B(-k)) U^H) / 2 (symmetry.py:78-86).  -k is the "mod" index
// (-i mod n) or the "flip" index (n - 1 - i) along the selected axes
// (symmetry.py:18-41).  One CTA per k-point holds A and the products in
// shared memory; group elements are read from global memory (they are shared
// by every k and stay in L1/L2).
#include "common.cuh"

#include <algorithm>

namespace cpphf {

namespace {

constexpr int kSymThreads = 256;
constexpr int kSymMaxNb = 64;

__device__ __forceinline__ int64_t minus_k(int64_t k, int nk1, int nk2, int conv, int axes) {
    const int i = (int)(k / nk2), j = (int)(k - (int64_t)(k / nk2) * nk2);
    int mi = i, mj = j;
    if (axes & 1) mi = conv == 0 ? (nk1 - i) % nk1 : nk1 - 1 - i;
    if (axes & 2) mj = conv == 0 ? (nk2 - j) % nk2 : nk2 - 1 - j;
    return (int64_t)mi * nk2 + mj;
}

// acc += sum over the group elements of g X g^H, X already in sA
__device__ void conj_sum(const double2* __restrict__ Gp, int ng, const double2* sA, double2* sX, double2* sAcc,
                         int nb) {
    const int nb2 = nb * nb;
    for (int g = 0; g < ng; ++g) {
        const double2* G = Gp + (size_t)g * nb2;
        for (int e = threadIdx.x; e < nb2; e += blockDim.x) {  // X = g A
            const int i = e / nb, m = e - i * nb;
            double2 acc = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) cfma(acc, G[i * nb + l], sA[l * nb + m]);
            sX[e] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nb2; e += blockDim.x) {  // acc += X g^H
            const int i = e / nb, j = e - i * nb;
            double2 acc = mk(0.0, 0.0);
            for (int m = 0; m < nb; ++m) cfma(acc, sX[i * nb + m], cconj(G[j * nb + m]));
            sAcc[e] = cadd(sAcc[e], acc);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSymThreads) k_sym_group(const double2* __restrict__ A, double2* __restrict__ out,
                                                           const double2* __restrict__ G1, int n1,
                                                           const double2* __restrict__ G2, int n2, int nb, int nk1,
                                                           int nk2, int conv, int axes, double N) {
    extern __shared__ __align__(16) double2 sm[];
    const int nb2 = nb * nb;
    double2* sA = sm;
    double2* sX = sm + nb2;
    double2* sAcc = sm + 2 * nb2;
    const int64_t nk = (int64_t)nk1 * nk2;
    for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
        for (int e = threadIdx.x; e < nb2; e += blockDim.x) {
            sA[e] = A[(size_t)k * nb2 + e];
            sAcc[e] = mk(0.0, 0.0);
        }
        __syncthreads();
        conj_sum(G1, n1, sA, sX, sAcc, nb);
        if (n2 > 0) {
            const int64_t km = minus_k(k, nk1, nk2, conv, axes);
            for (int e = threadIdx.x; e < nb2; e += blockDim.x) sA[e] = A[(size_t)km * nb2 + e];
            __syncthreads();
            conj_sum(G2, n2, sA, sX, sAcc, nb);
        }
        for (int e = threadIdx.x; e < nb2; e += blockDim.x) {
            const double2 v = sAcc[e];
            out[(size_t)k * nb2 + e] = mk(v.x / N, v.y / N);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSymThreads) k_sym_time_reversal(const double2* __restrict__ B,
                                                                   double2* __restrict__ out,
                                                                   const double2* __restrict__ U, int nb, int nk1,
                                                                   int nk2, int conv, int axes) {
    extern __shared__ __align__(16) double2 sm[];
    const int nb2 = nb * nb;
    double2* sB = sm;
    double2* sX = sm + nb2;
    const int64_t nk = (int64_t)nk1 * nk2;
    for (int64_t k = blockIdx.x; k < nk; k += gridDim.x) {
        const int64_t km = minus_k(k, nk1, nk2, conv, axes);
        for (int e = threadIdx.x; e < nb2; e += blockDim.x) sB[e] = cconj(B[(size_t)km * nb2 + e]);
        __syncthreads();
        for (int e = threadIdx.x; e < nb2; e += blockDim.x) {  // X = U conj(B(-k))
            const int i = e / nb, m = e - i * nb;
            double2 acc = mk(0.0, 0.0);
            for (int l = 0; l < nb; ++l) cfma(acc, U[i * nb + l], sB[l * nb + m]);
            sX[e] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < nb2; e += blockDim.x) {  // (B + X U^H) / 2
            const int i = e / nb, j = e - i * nb;
            double2 acc = mk(0.0, 0.0);
            for (int m = 0; m < nb; ++m) cfma(acc, sX[i * nb + m], cconj(U[j * nb + m]));
            const double2 b = B[(size_t)k * nb2 + e];
            out[(size_t)k * nb2 + e] = mk(0.5 * (b.x + acc.x), 0.5 * (b.y + acc.y));
        }
        __syncthreads();
    }
}

unsigned sym_grid(int64_t nk) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(nk, 8 * (int64_t)num_sms()));
}

}  // namespace

int symmetry_project(const cpphf_symmetry* s, double2* M, int64_t nk1, int64_t nk2, int64_t nb, cudaStream_t st) {
    if (!s || !M) return fail(CPPHF_ERR_INVALID, "symmetry_project: null pointer");
    if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(CPPHF_ERR_INVALID, "symmetry_project: empty field");
    if (nb > kSymMaxNb) return fail(CPPHF_ERR_UNSUPPORTED, "symmetry_project: nb above 64 is not supported");
    const bool group = s->n_unitary > 0 || s->n_spatial > 0;
    const bool tr = s->time_reversal_U != nullptr;
    if (!group && !tr) return CPPHF_OK;
    if (s->n_unitary > 0 && !s->unitary_group) return fail(CPPHF_ERR_INVALID, "symmetry_project: null unitary group");
    if (s->n_spatial > 0 && !s->spatial_group) return fail(CPPHF_ERR_INVALID, "symmetry_project: null spatial group");
    if (!s->scratch) return fail(CPPHF_ERR_INVALID, "symmetry_project: null scratch field");
    for (int c : {s->spatial_convention, s->tr_convention})
        if (c != 0 && c != 1) return fail(CPPHF_ERR_INVALID, "k_convention must be 'mod' or 'flip'");
    static bool attrs = [] {
        cudaFuncSetAttribute(k_sym_group, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(3 * sizeof(double2) * kSymMaxNb * kSymMaxNb));
        cudaFuncSetAttribute(k_sym_time_reversal, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * sizeof(double2) * kSymMaxNb * kSymMaxNb));
        (void)cudaGetLastError();
        return true;
    }();
    (void)attrs;
    const int64_t nk = nk1 * nk2;
    const size_t fbytes = sizeof(double2) * (size_t)nk * nb * nb;
    double2* scratch = static_cast<double2*>(s->scratch);
    const size_t m2 = sizeof(double2) * (size_t)nb * nb;
    if (group) {
        // a spatial group alone averages with the identity on A(k) (symmetry.py:106-108);
        // the caller passes that identity as the one-element unitary group
        const double N = (double)(s->n_unitary + s->n_spatial);
        k_sym_group<<<sym_grid(nk), kSymThreads, 3 * m2, st>>>(
            M, scratch, static_cast<const double2*>(s->unitary_group), (int)s->n_unitary,
            static_cast<const double2*>(s->spatial_group), (int)s->n_spatial, (int)nb, (int)nk1, (int)nk2,
            s->spatial_convention, s->spatial_axes, N);
        CPPHF_LAUNCH_CHECK("symmetry group average");
        if (!tr) {
            CPPHF_CUDA(cudaMemcpyAsync(M, scratch, fbytes, cudaMemcpyDeviceToDevice, st));
            return CPPHF_OK;
        }
    } else {
        CPPHF_CUDA(cudaMemcpyAsync(scratch, M, fbytes, cudaMemcpyDeviceToDevice, st));
    }
    k_sym_time_reversal<<<sym_grid(nk), kSymThreads, 2 * m2, st>>>(scratch, M,
                                                                   static_cast<const double2*>(s->time_reversal_U),
                                                                   (int)nb, (int)nk1, (int)nk2, s->tr_convention,
                                                                   s->tr_axes);
    CPPHF_LAUNCH_CHECK("symmetry time reversal");
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" {

int cpphf_symmetry_project(const cpphf_symmetry* sym, void* M, int64_t nk1, int64_t nk2, int64_t nb, void* stream) {
    return cpphf::symmetry_project(sym, static_cast<double2*>(M), nk1, nk2, nb, static_cast<cudaStream_t>(stream));
}

int cpphf_symmetry_project_fn(void* user, void* M, int64_t nk1, int64_t nk2, int64_t nb, void* stream) {
    return cpphf::symmetry_project(static_cast<const cpphf_symmetry*>(user), static_cast<double2*>(M), nk1, nk2, nb,
                                   static_cast<cudaStream_t>(stream));
}

}  // extern "C"
