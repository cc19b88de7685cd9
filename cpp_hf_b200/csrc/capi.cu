// Library-wide C-ABI plumbing: version, thread-local error text, SM count.
#include "common.cuh"

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

int num_sms() {
    int dev = 0;
    cudaGetDevice(&dev);
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

}  // namespace cpphf

extern "C" {

const char* cpphf_last_error(void) { return cpphf::g_last_error.c_str(); }

int cpphf_version(void) { return CPPHF_ABI_VERSION; }

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
