// Shared device/host helpers for the cpp_hf B200 library: complex arithmetic on
// double2/float2, status codes, the thread-local error message, launch checks
// and a bounded grid barrier for cooperative persistent kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/cpphf_b200.h"

namespace cpphf {

// ---------------------------------------------------------------------------
// Error reporting
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);

#define CPPHF_CUDA(call)                                              \
    do {                                                              \
        cudaError_t e__ = (call);                                     \
        if (e__ != cudaSuccess) return ::cpphf::cuda_fail(e__, #call); \
    } while (0)

#define CPPHF_LAUNCH_CHECK(name)                                      \
    do {                                                              \
        cudaError_t e__ = cudaGetLastError();                         \
        if (e__ != cudaSuccess) return ::cpphf::cuda_fail(e__, name); \
    } while (0)

#define CPPHF_TRY(call)                     \
    do {                                    \
        int s__ = (call);                   \
        if (s__ != CPPHF_OK) return s__;    \
    } while (0)

int num_sms();

// ---------------------------------------------------------------------------
// Device error word.  One per device (a __device__ variable of capi.cu): a
// bounded wait that gives up ORs a code into it, the kernel returns, and the
// host learns of it when it next reads the word (check_wait_error(), which
// synchronises the stream, or cpphf_device_error()).  Launches with bounded
// waits receive its address in their arguments.
// ---------------------------------------------------------------------------
constexpr unsigned kWaitErrMbar = 1u;     // an mbarrier (TMA / bulk copy) wait
constexpr unsigned kWaitErrBarrier = 2u;  // a grid barrier of a cooperative kernel

// Address of the current device's error word (nullptr and the error text set
// if it cannot be looked up).
unsigned* wait_error_word();
// Synchronise `st`, read the current device's error word and clear it; a set
// word returns CPPHF_ERR_TIMEOUT with `where` in the message.
int check_wait_error(cudaStream_t st, const char* where);
// Grid-barrier poll limit in force (cpphf_set_barrier_spin_limit).
long long barrier_spin_limit();

// Raise a kernel's dynamic shared-memory limit to the device opt-in maximum
// minus its static shared memory.  Attribute calls never leave a sticky error.
template <class F>
inline void raise_smem(F f) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, f) == cudaSuccess) {
        const int want = optin - (int)fa.sharedSizeBytes;
        if (want > 0) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, want);
    }
    (void)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Complex arithmetic
// ---------------------------------------------------------------------------
template <class R> struct CT;
template <> struct CT<double> { using type = double2; };
template <> struct CT<float> { using type = float2; };

__host__ __device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }

template <class C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <class C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <class C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <class C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <class C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
template <class C, class R> __host__ __device__ __forceinline__ C cscale(C a, R s) { return mk(a.x * s, a.y * s); }
// multiply by +i (s=+1) or -i (s=-1)
template <int S, class C> __host__ __device__ __forceinline__ C cmuli(C a) {
    return S > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
// acc += a * b
template <class C> __host__ __device__ __forceinline__ void cfma(C& acc, C a, C b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
// acc += a * conj(b)
template <class C> __host__ __device__ __forceinline__ void cfmac(C& acc, C a, C b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.y, b.x, acc.y);
    acc.y = fma(-a.x, b.y, acc.y);
}
__device__ __forceinline__ float2 to_c(double2 a, float2) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_c(double2 a, double2) { return a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }

// Streaming (evict-first) and L2-only loads/stores for read-once and
// intermediate fields.
__device__ __forceinline__ double2 ld_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ double2 ld_l2(const double2* p) { return __ldcg(p); }
__device__ __forceinline__ void st_l2(double2* p, double2 v) { __stcg(p, v); }
__device__ __forceinline__ float2 ld_l2(const float2* p) { return __ldcg(p); }
__device__ __forceinline__ void st_l2(float2* p, float2 v) { __stcg(p, v); }

// Kahan-compensated per-thread accumulator (a thread's long serial chain of
// terms); the cross-thread sums that follow are short fixed trees.
struct Kahan {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        const double y = x - c;
        const double t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

// ---------------------------------------------------------------------------
// Warp / block reductions (fixed order -> deterministic)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum NV values per thread over the block; result valid in every thread.
// `scratch` holds at least 32*NV doubles (checked at compile time).  Fixed
// reduction tree -> bitwise reproducible.
template <int NV, int M>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (&scratch)[M]) {
    static_assert(M >= 32 * NV, "block_sum scratch needs 32 doubles per value");
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) scratch[i * 32 + wid] = v[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double s = (lane < nw) ? scratch[i * 32 + lane] : 0.0;
        v[i] = warp_sum(s);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Bounded grid barrier for cooperative launches.  `sync[0]` = arrival count,
// `sync[1]` = generation, `sync[2]` = error flag; zeroed before the launch.
// A wait that exceeds the poll limit sets the flag (and kWaitErrBarrier in the
// device error word), every block waiting on the barrier sees the flag and
// returns, and every later barrier returns at once, so no block waits forever.
// The limit is a launch argument (default kBarrierSpinLimit, settable through
// cpphf_set_barrier_spin_limit).
// ---------------------------------------------------------------------------
constexpr long long kBarrierSpinLimit = 20000000LL;  // polls (each an L2 round trip) -> seconds
#ifndef CPPHF_POLL_SLEEP_NS
#define CPPHF_POLL_SLEEP_NS 0
#endif
constexpr unsigned kPollSleepNs = CPPHF_POLL_SLEEP_NS;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

struct GridBarrier {
    unsigned* sync;
    unsigned* err;
    long long limit;
    unsigned gen;
    __device__ void init(unsigned* s, long long spin_limit, unsigned* err_word) {
        sync = s;
        err = err_word;
        limit = spin_limit;
        gen = 0;
    }
    __device__ void give_up() {
        atomicExch(&sync[2], 1u);
        if (err) atomicOr(err, kWaitErrBarrier);
    }
    // Returns false if the barrier failed (timeout seen anywhere).
    __device__ bool wait() {
        __syncthreads();
        __shared__ int ok_sh;
        if (threadIdx.x == 0) {
            int ok = 1;
            if (ld_acquire_u32(&sync[2]) != 0u) {
                ok = 0;
            } else {
                __threadfence();
                const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
                const unsigned arrived = atomicAdd(&sync[0], 1u);
                if (arrived == nblocks - 1) {
                    atomicExch(&sync[0], 0u);
                    __threadfence();
                    atomicAdd(&sync[1], 1u);
                } else {
                    long long spins = 0;
                    while (ld_acquire_u32(&sync[1]) == gen) {
                        if (ld_acquire_u32(&sync[2]) != 0u) { ok = 0; break; }
                        if (++spins > limit) {
                            give_up();
                            ok = 0;
                            break;
                        }
                        if (kPollSleepNs) __nanosleep(kPollSleepNs);
                    }
                }
                __threadfence();
            }
            gen += 1;
            ok_sh = ok;
        }
        __syncthreads();
        return ok_sh != 0;
    }
};

}  // namespace cpphf
