// Library-wide C-ABI plumbing: version, thread-local error text, SM count.
#include "common.cuh"
#include "bulk.cuh"

#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>
#include <string>

namespace cpphf {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

int cuda_fail(cudaError_t e, const char* where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return CPPHF_ERR_CUDA;
}

// The device error word (one object per device: this is the only translation
// unit that defines it; other units receive its address).
__device__ unsigned g_wait_error = 0;

namespace {
constexpr int kMaxDevices = 64;
std::atomic<long long> g_barrier_spin_limit{kBarrierSpinLimit};
}  // namespace

unsigned* wait_error_word() {
    static std::mutex mtx;
    static unsigned* ptrs[kMaxDevices] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        (void)cudaGetLastError();
        set_error("device error word: no usable current device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mtx);
    if (!ptrs[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_wait_error) != cudaSuccess) {
            cuda_fail(cudaGetLastError(), "device error word lookup");
            return nullptr;
        }
        ptrs[dev] = static_cast<unsigned*>(p);
    }
    return ptrs[dev];
}

int check_wait_error(cudaStream_t st, const char* where) {
    unsigned* w = wait_error_word();
    if (!w) return CPPHF_ERR_CUDA;
    unsigned v = 0;
    CPPHF_CUDA(cudaMemcpyAsync(&v, w, sizeof(v), cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    if (v == 0) return CPPHF_OK;
    CPPHF_CUDA(cudaMemsetAsync(w, 0, sizeof(unsigned), st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    std::string what = (v & kWaitErrBarrier) ? "a grid barrier" : "";
    if (v & kWaitErrMbar) what += what.empty() ? "an asynchronous-copy wait" : " and an asynchronous-copy wait";
    return fail(CPPHF_ERR_TIMEOUT, std::string(where) + ": " + what + " on the device gave up (bounded wait timeout)");
}

long long barrier_spin_limit() { return g_barrier_spin_limit.load(std::memory_order_relaxed); }

int num_sms() {
    int dev = 0;
    cudaGetDevice(&dev);
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

bool make_tensor_map_3d(CUtensorMap* map, const void* base, CUtensorMapDataType dt, unsigned long long d0,
                        unsigned long long d1, unsigned long long d2, unsigned long long stride1_bytes,
                        unsigned long long stride2_bytes, unsigned b0, unsigned b1, unsigned b2) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        (void)cudaGetLastError();
    });
    if (!encode) return false;
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {stride1_bytes, stride2_bytes};
    const cuuint32_t box[3] = {b0, b1, b2};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = encode(map, dt, 3, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace cpphf

extern "C" {

const char* cpphf_last_error(void) { return cpphf::g_last_error.c_str(); }

int cpphf_version(void) { return CPPHF_ABI_VERSION; }

int cpphf_set_barrier_spin_limit(long long polls) {
    cpphf::g_barrier_spin_limit.store(polls > 0 ? polls : cpphf::kBarrierSpinLimit, std::memory_order_relaxed);
    return CPPHF_OK;
}

long long cpphf_barrier_spin_limit(void) { return cpphf::barrier_spin_limit(); }

int cpphf_device_error(int clear) {
    unsigned* w = cpphf::wait_error_word();
    if (!w) return CPPHF_ERR_CUDA;
    unsigned v = 0;
    CPPHF_CUDA(cudaDeviceSynchronize());
    CPPHF_CUDA(cudaMemcpy(&v, w, sizeof(v), cudaMemcpyDeviceToHost));
    if (clear && v) CPPHF_CUDA(cudaMemset(w, 0, sizeof(unsigned)));
    return (int)v;
}

}  // extern "C"

extern "C" {

// Host <-> device copies on a stream, synchronised before returning (used by
// host-side projector callbacks that must see and replace a device field).
int cpphf_copy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CPPHF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    return CPPHF_OK;
}

int cpphf_copy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CPPHF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    CPPHF_CUDA(cudaStreamSynchronize(st));
    return CPPHF_OK;
}

}  // extern "C"

