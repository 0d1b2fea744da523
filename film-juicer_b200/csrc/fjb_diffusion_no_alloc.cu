// fjb_diffusion_no_alloc.cu -- diffusion entry point that allocates nothing.
//
// fjb_diffusion builds the three PSF tables on the host and uploads them into a
// device buffer it allocates and frees on every call (and synchronises the stream
// in between). This variant is for hosts that cannot allocate device memory on
// their render path: the PSF tables live in one file-scope device array of fixed
// size, the tables are built on the device by a small kernel, and the call only
// enqueues two kernels on the caller's stream.
//
// Limits:
//  * The array holds three channels of (kMaxDiffusionRadius + 1) rows x 176 taps
//    (167 KiB), enough for radius <= 80 (the limit of the convolution kernel's shared
//    memory tile); a larger radius is rejected.
//  * The array is shared by every call on a device, so calls that can overlap (other
//    streams, other host threads) race on it. Order them on one stream or on the host.
//  * The build kernel writes every entry of the rows it uses, zero padding included,
//    so nothing has to start at zero.
//  * The device address of the array is looked up (cudaGetSymbolAddress) on the first
//    call made on each device, with that device current; make that first call before
//    any stream capture begins.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/juicer_b200.h"
#include "fjb_diffusion.h"
#include "fjb_launches.h"

namespace {

constexpr int kNoAllocMaxRadius = fjb::kMaxDiffusionRadius;
constexpr int kNoAllocMaxTaps = ((2 * kNoAllocMaxRadius + 1 + 15) / 16) * 16;
constexpr int kChannelFloats = (kNoAllocMaxRadius + 1) * kNoAllocMaxTaps;
constexpr int kBuildThreads = 512;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_psf_scratch[3 * kChannelFloats];

std::mutex g_setup_mutex;
float* g_psf_address[kMaxDevices] = {};

struct PsfBuild {
    double lambda_px[9];
    double weights[3][9];
    int radius, taps;
    float* rows; // 3 x kChannelFloats
};

__device__ __forceinline__ float psf_sample(const PsfBuild& b, int ch, int dx, int dy) {
    const double kTwoPi = 6.283185307179586476925286766559;
    const double rho = sqrt((double)dx * (double)dx + (double)dy * (double)dy);
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const double l = b.lambda_px[k];
        v += b.weights[ch][k] * exp(-rho / l) / (kTwoPi * l * l);
    }
    return (float)v;
}

// One CTA per channel: the FP64 sum of the (2r+1)^2 stored float samples (per-thread
// partials folded in a fixed order), then the normalised rows |dy| = 0..r.
__global__ void __launch_bounds__(kBuildThreads) psf_build_kernel(const __grid_constant__ PsfBuild b) {
    __shared__ double warp_sums[kBuildThreads / 32];
    __shared__ double total;
    const int ch = blockIdx.x;
    const int r = b.radius, d = 2 * r + 1;
    double part = 0.0;
    for (int i = threadIdx.x; i < d * d; i += kBuildThreads) {
        const int iy = i / d, ix = i - iy * d;
        part += (double)psf_sample(b, ch, ix - r, iy - r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kBuildThreads / 32; ++w) s += warp_sums[w];
        total = s;
    }
    __syncthreads();
    const double sum = total;
    float* rows = b.rows + (size_t)ch * kChannelFloats;
    for (int i = threadIdx.x; i < (r + 1) * b.taps; i += kBuildThreads) {
        const int dy = i / b.taps, ix = i - dy * b.taps;
        rows[i] = ix < d ? (float)((double)psf_sample(b, ch, ix - r, dy) / sum) : 0.0f;
    }
}

void put_error(FjErrorBuffer* error, const char* text) {
    if (!error) return;
    error->length = 0;
    if (!error->data || error->capacity == 0) return;
    size_t n = 0;
    while (text[n] && n + 1 < error->capacity) {
        error->data[n] = text[n];
        ++n;
    }
    error->data[n] = '\0';
    error->length = n;
}

FjStatus status(uint32_t category, FjErrorBuffer* error, const char* text) {
    put_error(error, text);
    return FjStatus{category, FJ_API_NONE, 0};
}

FjStatus cuda_failure(cudaError_t e, FjErrorBuffer* error, const char* where) {
    if (error && error->data && error->capacity > 0) {
        const int n = std::snprintf(error->data, error->capacity, "%s: %s", where, cudaGetErrorString(e));
        error->length = n < 0 ? 0 : ((size_t)n < error->capacity ? (size_t)n : error->capacity - 1);
    }
    return FjStatus{e == cudaErrorMemoryAllocation ? FJ_STATUS_ALLOCATION_FAILURE : FJ_STATUS_CUDA_FAILURE,
                    FJ_API_CUDA_RUNTIME, (int32_t)e};
}

// Device address of the PSF array on the current device, looked up once per device
// and kept for the life of the process. A cudaDeviceReset (or any other teardown of
// the device's primary context) invalidates it, so the library must not be called
// across one.
cudaError_t psf_scratch_address(float** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_psf_address[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_psf_scratch);
        if (e != cudaSuccess) return e;
        g_psf_address[dev] = static_cast<float*>(p);
    }
    *out = g_psf_address[dev];
    return cudaSuccess;
}

} // namespace

extern "C" FjStatus fjb_diffusion_no_alloc(const FjDiffusionComponents* components, int32_t radius_px,
                                           double scatter_fraction, const float* src_r, const float* src_g,
                                           const float* src_b, float* dst_r, float* dst_g, float* dst_b,
                                           ptrdiff_t stride, int32_t width, int32_t height, void* stream,
                                           FjErrorBuffer* error) {
    try {
        if (!components || !src_r || !src_g || !src_b || !dst_r || !dst_g || !dst_b)
            return status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (radius_px < 0 || radius_px > kNoAllocMaxRadius)
            return status(FJ_STATUS_UNSUPPORTED_INPUT, error,
                          "diffusion radius outside 0..80, the size of the static PSF scratch");
        if (width <= 0 || height <= 0) {
            put_error(error, "");
            return FjStatus{FJ_STATUS_SUCCESS, FJ_API_NONE, 0};
        }
        if (stride < width) return status(FJ_STATUS_UNSUPPORTED_INPUT, error, "stride below width");
        if (dst_r == src_r || dst_g == src_g || dst_b == src_b)
            return status(FJ_STATUS_UNSUPPORTED_INPUT, error, "diffusion output must not alias its input");
        if (!(scatter_fraction >= 0.0 && scatter_fraction <= 1.0))
            return status(FJ_STATUS_PREPARATION_FAILURE, error, "diffusion scatter fraction outside [0, 1]");
        PsfBuild b{};
        const double* w[3] = {components->red_weights, components->green_weights, components->blue_weights};
        for (int k = 0; k < 9; ++k) {
            const double l = components->lambda_px[k];
            if (!(l > 0.0) || !std::isfinite(l))
                return status(FJ_STATUS_PREPARATION_FAILURE, error, "diffusion lambda must be positive");
            b.lambda_px[k] = l;
        }
        // With non-negative weights the PSF peaks at rho = 0, so a finite, non-zero
        // float peak means every stored sample is finite and the sum is positive: the
        // normalisation the host builder checks after the fact.
        const double kTwoPi = 6.283185307179586476925286766559;
        for (int c = 0; c < 3; ++c) {
            double peak = 0.0;
            for (int k = 0; k < 9; ++k) {
                if (!std::isfinite(w[c][k]) || w[c][k] < 0.0)
                    return status(FJ_STATUS_PREPARATION_FAILURE, error,
                                  "diffusion weights must be finite and non-negative");
                b.weights[c][k] = w[c][k];
                peak += w[c][k] / (kTwoPi * b.lambda_px[k] * b.lambda_px[k]);
            }
            const float stored = (float)peak;
            if (!(std::isfinite(stored) && stored > 0.0f))
                return status(FJ_STATUS_PREPARATION_FAILURE, error, "diffusion PSF does not normalise");
        }
        float* rows = nullptr;
        cudaError_t e = psf_scratch_address(&rows);
        if (e != cudaSuccess) return cuda_failure(e, error, "diffusion PSF scratch set-up");
        b.radius = radius_px;
        b.taps = ((2 * radius_px + 1 + 15) / 16) * 16;
        b.rows = rows;
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        fjb::count_launch();
        psf_build_kernel<<<3, kBuildThreads, 0, s>>>(b);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_failure(e, error, "diffusion PSF build");
        const float* psf[3] = {rows, rows + kChannelFloats, rows + 2 * kChannelFloats};
        float* dst[3] = {dst_r, dst_g, dst_b};
        const float* src[3] = {src_r, src_g, src_b};
        e = fjb::launch_diffusion(psf, radius_px, b.taps, (float)scatter_fraction, dst, src, stride, width, height, s);
        if (e != cudaSuccess) return cuda_failure(e, error, "diffusion");
        put_error(error, "");
        return FjStatus{FJ_STATUS_SUCCESS, FJ_API_NONE, 0};
    } catch (...) {
        return status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_diffusion_no_alloc");
    }
}
