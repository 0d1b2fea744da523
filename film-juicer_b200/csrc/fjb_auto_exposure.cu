// fjb_auto_exposure.cu -- camera auto-exposure metering (a14), one launch.
//
// Restates src/Cuda/JuicerCudaAutoExposure.cu:63-141 (sample grid and metering
// weights), :266-300 (centre weight: Gaussian sigma 0.2 of the long edge), :314-407
// (FP64 weighted sums of the reconstructed raw mean), :462-520 (EV = -log2(Y / 1) ->
// scale). Median metering is rejected, as in the reference
// (src/Cuda/JuicerCudaExecutor.cpp:3145).
//
// B200 shape: one persistent launch of at most kMeterBlocks CTAs. Each CTA reduces
// its samples in FP64 (warp shuffles, then shared memory) and writes one partial; the
// last CTA to finish (atomic ticket) folds the partials in CTA order -- a fixed order,
// so the result is deterministic -- and writes the float scale. The scratch (partials
// + ticket) is caller-supplied device memory of meter_scratch_bytes().
#include <cuda_runtime.h>

#include "fjb_internal.h"
#include "fjb_pixel_math.cuh"
#include "fjb_launches.h"

namespace fjb {

namespace {

constexpr int kMeterThreads = 256;
constexpr int kLanes = 4;

__device__ __forceinline__ int preview_coordinate(int i, int preview, int source) {
    if (preview <= 0 || source <= 0) return 0;
    const long long num = (2LL * i + 1LL) * (long long)source;
    const int c = (int)(num / (2LL * preview));
    return min(source - 1, max(0, c));
}

__device__ __forceinline__ void meter_weights(int method, int x, int y, int w, int h, float lum, float out[kLanes]) {
    for (int l = 0; l < kLanes; ++l) out[l] = 0.0f;
    if (method == kMeterAverage || method == kMeterMedian) {
        out[0] = 1.0f;
        return;
    }
    const int maxDim = w > h ? w : h;
    const float invMax = maxDim > 0 ? 1.0f / (float)maxDim : 0.0f;
    if (method == kMeterCenterWeighted) {
        const float sigma = 0.2f;
        const float nx = ((float)x / (float)w) - 0.5f;
        const float normX = nx * (float)w * invMax;
        const float wx = expf(-(normX * normX) / (2.0f * sigma * sigma));
        const float ny = ((float)y / (float)h) - 0.5f;
        const float normY = ny * (float)h * invMax;
        const float wy = expf(-(normY * normY) / (2.0f * sigma * sigma));
        out[0] = wx * wy;
        return;
    }
    const float nx = (((float)x / (float)w) - 0.5f) * (float)w * invMax;
    const float ny = (((float)y / (float)h) - 0.5f) * (float)h * invMax;
    const float radius = sqrtf(nx * nx + ny * ny);
    if (method == kMeterPartial) {
        out[0] = radius < 0.15f ? 1.0f : 0.0f;
        out[3] = 1.0f;
    } else if (method == kMeterMatrix) {
        const int ch = h / 5, cw = w / 5;
        if (ch <= 0 || cw <= 0) return;
        const int row = y / ch, col = x / cw;
        if (row >= 5 || col >= 5) return;
        const float dy = ((float)row - 2.0f) / 2.0f;
        const float dx = ((float)col - 2.0f) / 2.0f;
        const float dist = sqrtf(dx * dx + dy * dy) / sqrtf(2.0f);
        out[0] = 0.5f * (1.0f + cosf(3.14159265358979323846f * dist));
    } else if (method == kMeterMultiZone) {
        if (radius >= 0.0f && radius < 0.05f) out[0] = 1.0f;
        else if (radius >= 0.05f && radius < 0.25f) out[1] = 1.0f;
        else if (radius >= 0.25f && radius < 0.50f) out[2] = 1.0f;
        out[3] = 1.0f;
    } else if (method == kMeterHighlightWeighted) {
        out[0] = lum * lum;
        out[3] = 1.0f;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kMeterThreads) meter_kernel(const __grid_constant__ PixelParams p, MeterSpec m,
                                                              double* partials, unsigned* ticket, float* scale) {
    const int total = m.preview_width * m.preview_height;
    double sy[kLanes] = {0, 0, 0, 0}, sw[kLanes] = {0, 0, 0, 0};
    const int srcW = m.meter_x2 - m.meter_x1, srcH = m.meter_y2 - m.meter_y1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int y = i / m.preview_width, x = i - y * m.preview_width;
        const int py = m.meter_y1 + preview_coordinate(y, m.preview_height, srcH);
        const int px = m.meter_x1 + preview_coordinate(x, m.preview_width, srcW);
        if (py < m.source_y1 || py >= m.source_y2 || px < m.source_x1 || px >= m.source_x2) continue;
        const float* s = reinterpret_cast<const float*>(p.src + (long long)(py - m.source_y1) * p.src_row_bytes) +
                         (long long)(px - m.source_x1) * p.components;
        const float in[3] = {s[0], s[1], s[2]};
        float raw[3];
        if (p.method == kMallett) {
            mallett_exposure(p, in, raw);
        } else {
            float xyz[3];
            working_xyz(p, in, xyz);
            tc_exposure(p, xyz, raw);
        }
        const float mean = (raw[0] + raw[1] + raw[2]) * (1.0f / 3.0f);
        if (!isfinite(mean)) continue;
        float w[kLanes];
        meter_weights(m.method, x, y, m.preview_width, m.preview_height, mean, w);
        for (int l = 0; l < kLanes; ++l) {
            const float wl = (isfinite(w[l]) && w[l] > 0.0f) ? w[l] : 0.0f;
            sy[l] += (double)mean * (double)wl;
            sw[l] += (double)wl;
        }
    }
    __shared__ double red[kMeterThreads / 32][2 * kLanes];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int l = 0; l < kLanes; ++l) {
        const double a = warp_sum(sy[l]);
        const double b = warp_sum(sw[l]);
        if (lane == 0) {
            red[warp][l] = a;
            red[warp][kLanes + l] = b;
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * kLanes) {
        double acc = 0.0;
        for (int w = 0; w < kMeterThreads / 32; ++w) acc += red[w][threadIdx.x];
        partials[blockIdx.x * 2 * kLanes + threadIdx.x] = acc;
    }
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        double Y[kLanes] = {0, 0, 0, 0}, W[kLanes] = {0, 0, 0, 0};
        for (unsigned b = 0; b < gridDim.x; ++b) {
            const volatile double* q = partials + b * 2 * kLanes;
            for (int l = 0; l < kLanes; ++l) {
                Y[l] += q[l];
                W[l] += q[kLanes + l];
            }
        }
        double yexp = 0.0;
        bool has = false;
        if (m.method == kMeterPartial) {
            const int l = W[0] > 0.0 ? 0 : 3;
            if (W[l] > 0.0) {
                yexp = Y[l] / W[l];
                has = true;
            }
        } else if (m.method == kMeterMultiZone) {
            const double ring[3] = {0.50, 0.30, 0.20};
            double ws = 0.0, wt = 0.0;
            for (int l = 0; l < 3; ++l) {
                if (W[l] > 0.0) {
                    ws += ring[l] * Y[l] / W[l];
                    wt += ring[l];
                }
            }
            if (wt > 0.0) {
                yexp = ws / wt;
                has = true;
            } else if (W[3] > 0.0) {
                yexp = Y[3] / W[3];
                has = true;
            }
        } else if (m.method == kMeterHighlightWeighted && W[0] < 1e-12) {
            if (W[3] > 0.0) {
                yexp = Y[3] / W[3];
                has = true;
            }
        } else if (W[0] > 0.0) {
            yexp = Y[0] / W[0];
            has = true;
        }
        double ev = 0.0;
        if (has && isfinite(yexp) && yexp > 0.0) {
            const double c = -log(yexp / 1.0) / log(2.0);
            if (isfinite(c)) ev = c;
        }
        const double s64 = exp2(ev);
        *scale = (isfinite(s64) && s64 > 0.0) ? (float)s64 : 1.0f;
        *ticket = 0u; // ready for the next frame
    }
}

} // namespace

size_t meter_scratch_bytes() { return (size_t)kMeterBlocks * 2 * kLanes * sizeof(double) + 256; }

cudaError_t launch_auto_exposure(const PixelParams& p, const MeterSpec& m, void* scratch, float* scale,
                                 cudaStream_t stream) {
    if (m.method == kMeterMedian) return cudaErrorNotSupported;
    const int total = m.preview_width * m.preview_height;
    if (total <= 0) return cudaErrorInvalidValue;
    int grid = (total + kMeterThreads - 1) / kMeterThreads;
    if (grid > kMeterBlocks) grid = kMeterBlocks;
    double* partials = static_cast<double*>(scratch);
    unsigned* ticket = reinterpret_cast<unsigned*>(static_cast<char*>(scratch) + (size_t)kMeterBlocks * 2 * kLanes *
                                                                                      sizeof(double));
    fjb::count_launch();
    meter_kernel<<<grid, kMeterThreads, 0, stream>>>(p, m, partials, ticket, scale);
    return cudaGetLastError();
}

} // namespace fjb
