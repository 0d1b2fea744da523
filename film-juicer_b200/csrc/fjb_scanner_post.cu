// fjb_scanner_post.cu -- scanner post effects on linear output-RGB planes.
//
// Restates src/Cuda/Scan/JuicerCudaScanPipeline.cu of the reference:
//   glare      :273-316  per-pixel lognormal glare percent from a Box-Muller normal of the
//                        Philox stream (seed, absolute x, medium, absolute y), :214-256;
//   blurs      :318-446  separable Gaussian, half-sample reflection repeated as needed
//                        (:258-270), taps summed in order in FP64, stored as float
//                        (0 when not finite);
//   unsharp    :586-655  vertical pass of the horizontally blurred plane combined as
//                        v + amount (v - blurred) in FP64;
//   schedule   :2586-2878 glare (+ its blur) before the scan to linear RGB, then lens blur
//                        and unsharp per plane, then output encoding.
// Planes are dense (width floats per row). The blurs read their inputs through L1
// (typical radii are a few pixels); arithmetic order and rounding points follow the
// reference so results match it to the last bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "fjb_launches.h"
#include "fjb_philox.cuh"
#include "fjb_scanner_post.h"

namespace fjb {

namespace {

__device__ __forceinline__ int reflect_wide(long long i, int n) {
    if (n <= 1) return 0;
    while (i < 0 || i >= n) i = i < 0 ? -i - 1 : 2LL * n - i - 1;
    return (int)i;
}

__device__ __forceinline__ bool finite_d(double v) { return isfinite(v) && !isnan(v); }
__device__ __forceinline__ bool finite_f(float v) { return isfinite(v) && !isnan(v); }

__global__ void glare_kernel(float* out, int width, int height, uint64_t seed, uint32_t medium, int origin_x,
                             int origin_y, float percent, float roughness) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    const float mean = fmaxf(0.0f, percent);
    const float stddev = fmaxf(0.0f, roughness * percent);
    const uint64_t ax = (uint64_t)((int64_t)origin_x + (int64_t)x);
    const uint64_t ay = (uint64_t)((int64_t)origin_y + (int64_t)y);
    Philox rng(seed, (uint32_t)ax, medium, (uint32_t)ay);
    float u1 = philox_u01(rng.next());
    u1 = fminf(fmaxf(u1, 1e-7f), 1.0f);
    const float u2 = philox_u01(rng.next());
    const float r = sqrtf(-2.0f * logf(u1));
    constexpr float kTwoPi = 6.28318530717958647692f;
    const float n = r * cosf(kTwoPi * u2);
    // lognormal with the given mean and standard deviation
    const float m2 = mean * mean;
    const float s2 = stddev * stddev;
    const float sigmaSq = logf(1.0f + (s2 / m2));
    const float sigma = sqrtf(fmaxf(0.0f, sigmaSq));
    const float mu = logf(fmaxf(1e-12f, mean)) - 0.5f * sigmaSq;
    const float glare = expf(mu + sigma * n);
    out[(size_t)y * width + x] = finite_f(glare) ? glare : 0.0f;
}

__global__ void blur_rows_kernel(const float* __restrict__ in, float* __restrict__ out, int width, int height,
                                 const float* __restrict__ w, int radius) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    const float* row = in + (size_t)y * width;
    double acc = 0.0;
    const int n = 2 * radius + 1;
    for (int k = 0; k < n; ++k) {
        const float v = __ldg(row + reflect_wide((long long)x - radius + k, width));
        acc += (double)v * (double)__ldg(w + k);
    }
    out[(size_t)y * width + x] = finite_d(acc) ? (float)acc : 0.0f;
}

// Vertical pass; with `unsharp`, `io` holds the plane and receives
// v + amount (v - blurred); otherwise the blurred value goes to `io`.
template <bool kUnsharp>
__global__ void blur_cols_kernel(const float* __restrict__ in, float* io, int width, int height,
                                 const float* __restrict__ w, int radius, float amount) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    double acc = 0.0;
    const int n = 2 * radius + 1;
    for (int k = 0; k < n; ++k) {
        const float v = __ldg(in + (size_t)reflect_wide((long long)y - radius + k, height) * width + x);
        acc += (double)v * (double)__ldg(w + k);
    }
    const float blurred = finite_d(acc) ? (float)acc : 0.0f;
    const size_t idx = (size_t)y * width + x;
    if (kUnsharp) {
        const double v0 = (double)io[idx];
        const double vb = (double)blurred;
        const double a = (double)amount;
        const double o = v0 + a * (v0 - vb);
        io[idx] = finite_d(o) ? (float)o : 0.0f;
    } else {
        io[idx] = blurred;
    }
}

dim3 plane_grid(int width, int height) { return dim3((width + 31) / 32, (height + 7) / 8); }

} // namespace

cudaError_t launch_glare(float* out, int width, int height, uint64_t seed, uint32_t medium, int origin_x,
                         int origin_y, float percent, float roughness, cudaStream_t stream) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    fjb::count_launch();
    glare_kernel<<<plane_grid(width, height), dim3(32, 8), 0, stream>>>(out, width, height, seed, medium, origin_x,
                                                                       origin_y, percent, roughness);
    return cudaGetLastError();
}

cudaError_t launch_blur_plane(float* plane, float* tmp, int width, int height, const float* w, int radius,
                              cudaStream_t stream) {
    if (width <= 0 || height <= 0 || radius <= 0 || !w) return cudaSuccess;
    fjb::count_launch();
    blur_rows_kernel<<<plane_grid(width, height), dim3(32, 8), 0, stream>>>(plane, tmp, width, height, w, radius);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    fjb::count_launch();
    blur_cols_kernel<false><<<plane_grid(width, height), dim3(32, 8), 0, stream>>>(tmp, plane, width, height, w,
                                                                                   radius, 0.0f);
    return cudaGetLastError();
}

cudaError_t launch_unsharp_plane(float* plane, float* tmp, int width, int height, const float* w, int radius,
                                 float amount, cudaStream_t stream) {
    if (width <= 0 || height <= 0 || radius <= 0 || !w) return cudaSuccess;
    fjb::count_launch();
    blur_rows_kernel<<<plane_grid(width, height), dim3(32, 8), 0, stream>>>(plane, tmp, width, height, w, radius);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    fjb::count_launch();
    blur_cols_kernel<true><<<plane_grid(width, height), dim3(32, 8), 0, stream>>>(tmp, plane, width, height, w,
                                                                                  radius, amount);
    return cudaGetLastError();
}

} // namespace fjb
