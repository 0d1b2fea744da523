// fjb_highlight_boost.cu -- highlight reconstruction on the camera carrier planes.
//
// Restates src/Cuda/Film/JuicerCudaHighlightBoost.cu of the reference: the frame
// maximum over the three carrier planes (any negative or non-finite sample makes the
// carrier invalid), then, when the maximum exceeds the protection level, every sample
// above it is lifted along a normalised exponential curve so that the maximum lands on
// maximum * peak_gain. The FP64 preparation of the curve's parameters (:75-128) and the
// FP32 double-word evaluation per sample (:130-196) follow the reference step for step:
// they are the algorithm its tests pin.
//
// B200 schedule: one reduction launch (warp and block maxima, then one atomic max on the
// float bits -- non-negative floats order as unsigned integers -- and an atomic or of the
// invalid flag; a maximum does not depend on the order it is taken in), then one apply
// launch whose CTAs each derive the parameters from the maximum in shared memory (CTA 0
// also publishes the disposition for the host). The reference uses three launches and a
// per-block partials array.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "fjb_highlight_boost.h"
#include "fjb_launches.h"

namespace fjb {

namespace {

constexpr int kThreads = 256;

struct BoostParams {
    int disposition;
    float maximum, protection, protectionResidual, onset, peak, peakResidual, range, rangeResidual, shape,
        shapeResidual, tailExpFactor, tailLinearFactor, delta, inverseShapeNormalization;
};

__device__ __forceinline__ void take(float v, float& mx, unsigned& invalid) {
    if (isfinite(v) && v >= 0.0f)
        mx = fmaxf(mx, v);
    else
        invalid = 1u;
}

__global__ void __launch_bounds__(kThreads) boost_reduce_kernel(const float* __restrict__ b, const float* __restrict__ g,
                                                                const float* __restrict__ r, long long stride,
                                                                int width, long long pixels, BoostState* state) {
    float mx = 0.0f;
    unsigned invalid = 0u;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += step) {
        const long long row = i / width;
        const long long o = row * stride + (i - row * width);
        take(r[o], mx, invalid);
        take(g[o], mx, invalid);
        take(b[o], mx, invalid);
    }
    for (int s = 16; s > 0; s >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, s));
        invalid |= __shfl_xor_sync(0xffffffffu, invalid, s);
    }
    __shared__ float wmx[kThreads / 32];
    __shared__ unsigned winv[kThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        wmx[threadIdx.x >> 5] = mx;
        winv[threadIdx.x >> 5] = invalid;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) {
            mx = fmaxf(mx, wmx[w]);
            invalid |= winv[w];
        }
        atomicMax(&state->maximum_bits, __float_as_uint(mx));
        if (invalid) atomicOr(&state->invalid, 1u);
    }
}

// (exp(t) - t - 1) / t^2, extended at zero by its Taylor series (reference :66-73).
__device__ double normalized_exponential(double t) {
    if (t >= 0.03125) return (expm1(t) - t) / (t * t);
    return 0.5 + t * (1.0 / 6.0 + t * (1.0 / 24.0 + t * (1.0 / 120.0 + t * (1.0 / 720.0 +
               t * (1.0 / 5040.0 + t * (1.0 / 40320.0 + t * (1.0 / 362880.0 + t / 3628800.0)))))));
}

// FP64 preparation of the curve (reference :75-128).
__device__ void prepare(const BoostDescriptor& d, const BoostState& s, BoostParams& w) {
    w = BoostParams{};
    const float mx = __uint_as_float(s.maximum_bits);
    const double maximum = mx;
    w.maximum = mx;
    if (s.invalid != 0u) {
        w.disposition = kBoostInvalidCarrier;
        return;
    }
    if (maximum <= d.protection) {
        w.disposition = kBoostBypass;
        return;
    }
    const double peak = maximum * d.peak_gain;
    if (peak > (double)FLT_MAX) {
        w.disposition = kBoostPeakOverflow;
        return;
    }
    const double range = maximum - d.protection;
    const double shape = d.sharpness * range / maximum;
    const double normalization = normalized_exponential(shape);
    w.disposition = kBoostApplied;
    w.protection = __double2float_rn(d.protection);
    w.protectionResidual = __double2float_rn(d.protection - (double)w.protection);
    // strict onset: the first carrier float above the original double
    w.onset = (double)w.protection <= d.protection ? nextafterf(w.protection, __int_as_float(0x7f800000))
                                                   : w.protection;
    w.peak = __double2float_rn(peak);
    w.peakResidual = __double2float_rn(peak - (double)w.peak);
    w.range = __double2float_rn(range);
    w.rangeResidual = __double2float_rn(range - (double)w.range);
    w.shape = __double2float_rn(shape);
    w.shapeResidual = __double2float_rn(shape - (double)w.shape);
    if (w.shape >= 0.5f) {
        const double denominator = shape * shape * normalization;
        w.tailExpFactor = __double2float_rn(exp(shape) / denominator);
        w.tailLinearFactor = __double2float_rn(1.0 / denominator);
    }
    w.delta = __double2float_rn(maximum * (d.peak_gain - 1.0));
    w.inverseShapeNormalization = __double2float_rn(1.0 / normalization);
}

// FP32 normalised exponential of a double-word argument (reference :130-140).
__device__ float normalized_float(float t, float residual) {
    if (t < 0.5f) {
        return 0.5f + t * (1.0f / 6.0f + t * (1.0f / 24.0f + t * (1.0f / 120.0f + t * (1.0f / 720.0f +
                   t * (1.0f / 5040.0f + t * (1.0f / 40320.0f + t * (1.0f / 362880.0f + t / 3628800.0f)))))));
    }
    const float numerator = fmaf(expf(t), residual, expm1f(t) - t) - residual;
    return numerator / (t * t);
}

// One sample (reference :142-196): the fraction of the range above protection as a
// double word, the curve's ratio, and either the direct lift or, near the peak, the
// endpoint form that subtracts the remaining deficit from the peak.
__device__ float boost(float sample, const BoostParams& w) {
    if (sample < w.onset) return sample;
    if (sample == w.maximum) return w.peak;
    const float distance = sample - w.protection;
    const float virtualProtection = distance - sample;
    const float distanceResidual =
        ((sample - (distance - virtualProtection)) + (-w.protection - virtualProtection)) - w.protectionResidual;
    const float quotient = distance / w.range;
    const float correction =
        (fmaf(-quotient, w.range, distance) + distanceResidual - quotient * w.rangeResidual) / w.range;
    const float fraction = quotient + correction;
    const float virtualCorrection = fraction - quotient;
    const float fractionResidual = (quotient - (fraction - virtualCorrection)) + (correction - virtualCorrection);
    const float t = w.shape * fraction;
    const float tResidual = fmaf(w.shape, fraction, -t) + w.shape * fractionResidual + w.shapeResidual * fraction;
    const float fractionSquared = fmaf(2.0f * fraction, fractionResidual, fraction * fraction);
    const float ratio = fractionSquared * (normalized_float(t, tResidual) * w.inverseShapeNormalization);
    if (w.shape >= 0.5f && ratio >= 0.5f) {
        const float gap = w.maximum - sample;
        const float gapFraction = gap / w.range;
        const float gapResidual = (fmaf(-gapFraction, w.range, gap) - gapFraction * w.rangeResidual) / w.range;
        const float d = w.shape * gapFraction;
        const float dResidual = fmaf(w.shape, gapFraction, -d) + w.shape * gapResidual + w.shapeResidual * gapFraction;
        const float oneMinusExp = fmaf(expf(-d), dResidual, -expm1f(-d));
        const float tail = fmaf(oneMinusExp, w.tailExpFactor, -(d + dResidual) * w.tailLinearFactor);
        const float endpoint = w.peak - gap;
        const float virtualGap = w.peak - endpoint;
        const float endpointResidual = (w.peak - (endpoint + virtualGap)) + (virtualGap - gap);
        return endpoint + ((endpointResidual + w.peakResidual) - w.delta * tail);
    }
    return sample + w.delta * ratio;
}

__global__ void __launch_bounds__(kThreads) boost_apply_kernel(float* b, float* g, float* r, long long stride,
                                                               int width, long long pixels, BoostDescriptor d,
                                                               BoostState* state) {
    __shared__ BoostParams w;
    if (threadIdx.x == 0) {
        prepare(d, *state, w);
        if (blockIdx.x == 0) state->disposition = (unsigned)w.disposition;
    }
    __syncthreads();
    if (w.disposition != kBoostApplied) return;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += step) {
        const long long row = i / width;
        const long long o = row * stride + (i - row * width);
        r[o] = boost(r[o], w);
        g[o] = boost(g[o], w);
        b[o] = boost(b[o], w);
    }
}

} // namespace

cudaError_t launch_highlight_boost(const BoostDescriptor& d, float* b, float* g, float* r, long long stride, int width,
                                   int height, BoostState* state, cudaStream_t stream) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(state, 0, sizeof(BoostState), stream);
    if (e != cudaSuccess) return e;
    const long long pixels = (long long)width * height;
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const long long need = (pixels + kThreads - 1) / kThreads;
    const int grid = (int)(need < (long long)sms * 8 ? need : (long long)sms * 8);
    fjb::count_launch();
    boost_reduce_kernel<<<grid, kThreads, 0, stream>>>(b, g, r, stride, width, pixels, state);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    fjb::count_launch();
    boost_apply_kernel<<<grid, kThreads, 0, stream>>>(b, g, r, stride, width, pixels, d, state);
    return cudaGetLastError();
}

} // namespace fjb
