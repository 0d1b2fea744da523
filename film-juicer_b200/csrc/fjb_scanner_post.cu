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

// ---------------------------------------------------------------------------
// Run form of the blurs: a thread computes kRun consecutive outputs. Its inputs sit in
// a ring of kRun doubles (each converted once), every tap is converted once per run,
// and output j still sums its taps in order, starting from zero, so the results are
// those of the per-output loop above bit for bit.
// ---------------------------------------------------------------------------
constexpr int kRun = 9; // odd: threads nine samples apart read distinct shared-memory banks
constexpr int kTileThreads = 256;
constexpr int kTileRows = 2;
constexpr size_t kTileSmemLimit = 200 * 1024;

struct Planes {
    float* p[3];
};

// sum[j] = sum_o in(j + o) w[o], o = 0 .. n-1 in order; get(i) is input i of the run
// (get(i) for i up to n - 1 + kRun is evaluated).
template <typename Get>
__device__ __forceinline__ void run_taps(const float* __restrict__ w, int n, Get get, double (&sum)[kRun]) {
    double ring[kRun];
#pragma unroll
    for (int i = 0; i < kRun; ++i) {
        sum[i] = 0.0;
        ring[i] = (double)get(i);
    }
    for (int ob = 0; ob < n; ob += kRun) {
#pragma unroll
        for (int s = 0; s < kRun; ++s) {
            const int o = ob + s;
            if (o < n) {
                const double t = (double)__ldg(w + o);
#pragma unroll
                for (int j = 0; j < kRun; ++j) sum[j] += ring[(s + j) % kRun] * t;
                ring[s] = (double)get(o + kRun); // input o leaves the run, input o + kRun enters
            }
        }
    }
}

__host__ __device__ inline int tile_stride(int width, int radius) { return width + 2 * radius + kRun + 1; }

size_t tile_smem_bytes(int width, int radius) {
    return ((size_t)kTileRows * tile_stride(width, radius) + (size_t)(kTileThreads / 32) * 32 * kRun) * sizeof(float);
}

// Horizontal pass over kTileRows rows per CTA (plane blockIdx.y): each row, reflected
// out to the radius on both sides, in shared memory; outputs leave through a per-warp
// staging area so that the stores are coalesced.
__global__ void __launch_bounds__(kTileThreads) blur_rows_tile_kernel(const __grid_constant__ Planes in,
                                                                      const __grid_constant__ Planes out, int width, int height,
                                                                      const float* __restrict__ w, int radius) {
    extern __shared__ float tile[];
    const int stride = tile_stride(width, radius);
    const float* src = in.p[blockIdx.y];
    float* dst = out.p[blockIdx.y];
    const int y0 = blockIdx.x * kTileRows;
    const int rows = min(kTileRows, height - y0);
    for (int rr = 0; rr < rows; ++rr) {
        const float* row = src + (size_t)(y0 + rr) * width;
        for (int i = threadIdx.x; i < stride; i += blockDim.x) {
            const long long q = (long long)i - radius;
            float v = 0.0f;
            if (i < width + 2 * radius)
                v = __ldg(row + ((unsigned long long)q < (unsigned long long)width ? (int)q : reflect_wide(q, width)));
            tile[rr * stride + i] = v;
        }
    }
    __syncthreads();
    const int n = 2 * radius + 1, nb = (width + kRun - 1) / kRun, tasks = rows * nb;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    float* st = tile + kTileRows * stride + warp * 32 * kRun;
    for (int base = warp * 32; base < tasks; base += warps * 32) {
        const int task = base + lane;
        if (task < tasks) {
            const int rr = task / nb, p0 = (task - rr * nb) * kRun;
            const float* line = tile + rr * stride + p0;
            double sum[kRun];
            run_taps(w, n, [&](int i) { return line[i]; }, sum);
#pragma unroll
            for (int j = 0; j < kRun; ++j) st[lane * kRun + j] = finite_d(sum[j]) ? (float)sum[j] : 0.0f;
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kRun; ++i) {
            const int e = i * 32 + lane, tk = base + e / kRun;
            if (tk < tasks) {
                const int rr = tk / nb, x = (tk - rr * nb) * kRun + e % kRun;
                if (x < width) dst[(size_t)(y0 + rr) * width + x] = st[e];
            }
        }
        __syncwarp();
    }
}

// Vertical pass (plane blockIdx.z): a thread takes kRun rows of one column; the warp's
// loads are rows of 32 consecutive columns. With kUnsharp, `io` holds the plane and
// receives v + amount (v - blurred) in FP64; otherwise the blurred value goes to `io`.
template <bool kUnsharp>
__global__ void __launch_bounds__(256) blur_cols_run_kernel(const __grid_constant__ Planes in,
                                                            const __grid_constant__ Planes io, int width, int height,
                                                            const float* __restrict__ w, int radius, float amount) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int p0 = (blockIdx.y * blockDim.y + threadIdx.y) * kRun;
    if (x >= width || p0 >= height) return;
    const float* src = in.p[blockIdx.z];
    float* dst = io.p[blockIdx.z];
    double sum[kRun];
    run_taps(w, 2 * radius + 1, [&](int i) {
        const long long q = (long long)p0 - radius + i;
        const int y = (unsigned long long)q < (unsigned long long)height ? (int)q : reflect_wide(q, height);
        return __ldg(src + (size_t)y * width + x);
    }, sum);
#pragma unroll
    for (int j = 0; j < kRun; ++j) {
        const int y = p0 + j;
        if (y >= height) break;
        const float blurred = finite_d(sum[j]) ? (float)sum[j] : 0.0f;
        const size_t idx = (size_t)y * width + x;
        if (kUnsharp) {
            const double v0 = (double)dst[idx];
            const double vb = (double)blurred;
            const double a = (double)amount;
            const double o = v0 + a * (v0 - vb);
            dst[idx] = finite_d(o) ? (float)o : 0.0f;
        } else {
            dst[idx] = blurred;
        }
    }
}

dim3 plane_grid(int width, int height) { return dim3((width + 31) / 32, (height + 7) / 8); }

// Horizontal pass of `count` planes into `tmps`: the tile kernel when a tile fits in
// shared memory, else the per-output kernel.
cudaError_t blur_rows(float* const* planes, float* const* tmps, int count, int width, int height, const float* w,
                      int radius, cudaStream_t stream) {
    const size_t smem = tile_smem_bytes(width, radius);
    if (smem <= kTileSmemLimit) {
        Planes in{}, out{};
        for (int c = 0; c < count; ++c) {
            in.p[c] = planes[c];
            out.p[c] = tmps[c];
        }
        cudaError_t e = cudaFuncSetAttribute(blur_rows_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        fjb::count_launch();
        blur_rows_tile_kernel<<<dim3((height + kTileRows - 1) / kTileRows, count), kTileThreads, smem, stream>>>(
            in, out, width, height, w, radius);
        return cudaGetLastError();
    }
    for (int c = 0; c < count; ++c) {
        fjb::count_launch();
        blur_rows_kernel<<<plane_grid(width, height), dim3(32, 8), 0, stream>>>(planes[c], tmps[c], width, height, w,
                                                                               radius);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <bool kUnsharp>
cudaError_t blur_cols(float* const* planes, float* const* tmps, int count, int width, int height, const float* w,
                      int radius, float amount, cudaStream_t stream) {
    Planes in{}, io{};
    for (int c = 0; c < count; ++c) {
        in.p[c] = tmps[c];
        io.p[c] = planes[c];
    }
    const int runs = (height + kRun - 1) / kRun;
    fjb::count_launch();
    blur_cols_run_kernel<kUnsharp><<<dim3((width + 31) / 32, (runs + 7) / 8, count), dim3(32, 8), 0, stream>>>(
        in, io, width, height, w, radius, amount);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_glare(float* out, int width, int height, uint64_t seed, uint32_t medium, int origin_x,
                         int origin_y, float percent, float roughness, cudaStream_t stream) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    fjb::count_launch();
    glare_kernel<<<plane_grid(width, height), dim3(32, 8), 0, stream>>>(out, width, height, seed, medium, origin_x,
                                                                       origin_y, percent, roughness);
    return cudaGetLastError();
}

cudaError_t launch_blur_planes(float* const* planes, float* const* tmps, int count, int width, int height,
                               const float* w, int radius, cudaStream_t stream) {
    if (width <= 0 || height <= 0 || radius <= 0 || !w || count <= 0) return cudaSuccess;
    if (count > 3) return cudaErrorInvalidValue;
    cudaError_t e = blur_rows(planes, tmps, count, width, height, w, radius, stream);
    if (e != cudaSuccess) return e;
    return blur_cols<false>(planes, tmps, count, width, height, w, radius, 0.0f, stream);
}

cudaError_t launch_unsharp_planes(float* const* planes, float* const* tmps, int count, int width, int height,
                                  const float* w, int radius, float amount, cudaStream_t stream) {
    if (width <= 0 || height <= 0 || radius <= 0 || !w || count <= 0) return cudaSuccess;
    if (count > 3) return cudaErrorInvalidValue;
    cudaError_t e = blur_rows(planes, tmps, count, width, height, w, radius, stream);
    if (e != cudaSuccess) return e;
    return blur_cols<true>(planes, tmps, count, width, height, w, radius, amount, stream);
}

} // namespace fjb
