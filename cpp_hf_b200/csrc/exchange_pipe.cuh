// Shared-memory layout helpers and the list of register-codelet line lengths
// of the pipelined exchange passes (exchange.cu, fock_packed.cu).
#pragma once

#include "common.cuh"

namespace cpphf {

// Offsets are relative to a 128-byte aligned base (TMA tensor copies need
// 128-byte aligned shared-memory destinations); `total` includes the slack
// for aligning the dynamic shared-memory base.
constexpr int kMaxPipeStages = 4;
constexpr int kColsMaxThreads = 128;  // launch bound of the pipelined columns pass
constexpr size_t kSmemMax = 227 * 1024 - 1024;

struct PipeLayout {
    size_t tw, bar, stage0, stage_bytes, in_bytes, total;
};


__host__ __device__ inline PipeLayout pipe_layout(int N, int CB, size_t in_elem, bool second, int nst) {
    PipeLayout L;
    L.tw = 0;
    L.bar = (sizeof(double2) * (size_t)N + 15) & ~(size_t)15;
    L.stage0 = (L.bar + 8 * kMaxPipeStages + 127) & ~(size_t)127;
    L.in_bytes = ((in_elem * (size_t)N * CB) + 127) & ~(size_t)127;
    L.stage_bytes = L.in_bytes + (second ? sizeof(double2) * (size_t)N * CB : 0);
    L.stage_bytes = (L.stage_bytes + 127) & ~(size_t)127;
    L.total = L.stage0 + (size_t)nst * L.stage_bytes + 128;
    return L;
}

// 128-byte aligned start inside a dynamic shared-memory array.  The offset is
// taken from the 32-bit shared address and added to the array itself, so the
// result stays a shared-memory pointer (a round trip through uintptr_t would
// turn every access into a generic 64-bit one).
__device__ __forceinline__ unsigned char* align128(unsigned char* p) {
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
    return p + ((128u - (a & 127u)) & 127u);
}

// (N, N1, N2): line lengths N = N1 * N2 with register codelets
#define CPPHF_SPEC_SIZES(X) \
    X(1, 1, 1)              \
    X(2, 2, 1)              \
    X(3, 3, 1)              \
    X(4, 4, 1)              \
    X(5, 5, 1)              \
    X(6, 3, 2)              \
    X(8, 4, 2)              \
    X(9, 3, 3)              \
    X(12, 4, 3)             \
    X(16, 4, 4)             \
    X(18, 6, 3)             \
    X(24, 6, 4)             \
    X(32, 8, 4)             \
    X(36, 6, 6)             \
    X(48, 8, 6)             \
    X(64, 8, 8)             \
    X(72, 9, 8)             \
    X(96, 12, 8)            \
    X(128, 16, 8)           \
    X(144, 12, 12)          \
    X(192, 16, 12)          \
    X(256, 16, 16)          \
    X(288, 18, 16)

}  // namespace cpphf
