// Periodic linear resampling of a k-mesh field (nk_old, nk_old, inner) ->
// (nk_new, nk_new, inner) (cpp_hf utils.hpp:120-176, resample_kgrid_2d).
//
// The reference resamples axis 0, then axis 1 of the intermediate; along one
// axis output index j reads x at u = (j - n_new/2) * (n_old / n_new) + n_old/2
// (centred grids, k = 0 at index n/2), floor(u) modulo n_old and its periodic
// neighbour, with weights 1 - frac and frac.  One launch evaluates both
// passes per output element in the reference's order:
//   t0 = a0 x[i0][i1] + b0 x[i0'][i1],  t1 = a0 x[i0][i1'] + b0 x[i0'][i1'],
//   y  = a1 t0 + b1 t1,
// with separately rounded products and sums (no fused multiply-add), so the
// result is the two-pass one bit for bit.  Threads run over the inner index
// fastest, so every access is a coalesced row segment.
#include "common.cuh"

#include <algorithm>
#include <cmath>

namespace cpphf {

namespace {

struct AxisTap {
    int64_t i0, i1;
    double a, b;
};

__device__ __forceinline__ AxisTap axis_tap(int64_t j, int64_t n_old, int64_t n_new, double ratio) {
    const double u = __dadd_rn(__dmul_rn((double)(j - n_new / 2), ratio), (double)(n_old / 2));
    const double fl = floor(u);
    int64_t i0 = (int64_t)fl;
    i0 = ((i0 % n_old) + n_old) % n_old;
    AxisTap t;
    t.i0 = i0;
    t.i1 = (i0 + 1) % n_old;
    const double frac = __dsub_rn(u, fl);
    t.a = __dsub_rn(1.0, frac);
    t.b = frac;
    return t;
}

__device__ __forceinline__ double2 lerp2(double a, double2 x0, double b, double2 x1) {
    return mk(__dadd_rn(__dmul_rn(a, x0.x), __dmul_rn(b, x1.x)), __dadd_rn(__dmul_rn(a, x0.y), __dmul_rn(b, x1.y)));
}

__global__ void k_resample_2d(const double2* __restrict__ x, double2* __restrict__ y, int64_t n_old, int64_t n_new,
                              int64_t inner, double ratio) {
    const int64_t total = n_new * n_new * inner;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % inner;
        const int64_t jj = e / inner;
        const int64_t j1 = jj % n_new, j0 = jj / n_new;
        const AxisTap t0 = axis_tap(j0, n_old, n_new, ratio);
        const AxisTap t1 = axis_tap(j1, n_old, n_new, ratio);
        const size_t row = (size_t)n_old * inner;
        const double2* r0 = x + (size_t)t0.i0 * row;
        const double2* r1 = x + (size_t)t0.i1 * row;
        const double2 x00 = r0[(size_t)t1.i0 * inner + i], x10 = r1[(size_t)t1.i0 * inner + i];
        const double2 x01 = r0[(size_t)t1.i1 * inner + i], x11 = r1[(size_t)t1.i1 * inner + i];
        const double2 c0 = lerp2(t0.a, x00, t0.b, x10);  // intermediate at (j0, t1.i0)
        const double2 c1 = lerp2(t0.a, x01, t0.b, x11);  // intermediate at (j0, t1.i1)
        y[e] = lerp2(t1.a, c0, t1.b, c1);
    }
}

}  // namespace

int resample_kgrid_2d(const double2* x, double2* y, int64_t nk_old, int64_t nk_new, int64_t inner, cudaStream_t st) {
    if (nk_old < 1 || nk_new < 1 || inner < 1) return fail(CPPHF_ERR_INVALID, "resample_kgrid_2d: empty array");
    if (!x || !y) return fail(CPPHF_ERR_INVALID, "resample_kgrid_2d: null pointer");
    const int64_t total = nk_new * nk_new * inner;
    if (nk_old == nk_new) {
        CPPHF_CUDA(cudaMemcpyAsync(y, x, sizeof(double2) * (size_t)total, cudaMemcpyDeviceToDevice, st));
        return CPPHF_OK;
    }
    const double ratio = (double)nk_old / (double)nk_new;
    const int64_t want = (total + 255) / 256;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 32 * (int64_t)num_sms()));
    k_resample_2d<<<grid, 256, 0, st>>>(x, y, nk_old, nk_new, inner, ratio);
    CPPHF_LAUNCH_CHECK("resample_kgrid_2d");
    return CPPHF_OK;
}

}  // namespace cpphf

extern "C" int cpphf_resample_kgrid_2d(const void* values, void* out, int64_t nk_old, int64_t nk_new, int64_t inner,
                                       void* stream) {
    return cpphf::resample_kgrid_2d(static_cast<const double2*>(values), static_cast<double2*>(out), nk_old, nk_new,
                                    inner, static_cast<cudaStream_t>(stream));
}
