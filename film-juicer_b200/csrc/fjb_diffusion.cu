// fjb_diffusion.cu -- camera / enlarger diffusion filter (a17): a radially symmetric
// point spread function convolved with each carrier plane, mixed with the plane.
//
// Semantics restate src/Cuda/Diffusion/JuicerCudaDiffusion.cu:294-487: the PSF on
// the (2r+1)^2 grid is sum_k w_k exp(-rho / lambda_k) / (2 pi lambda_k^2) in FP64,
// stored as float and normalised by the FP64 sum of the stored floats; the frame is
// extended by whole-sample reflection (period 2(n-1)); the output is
// (1 - f) x + f (PSF * x). The reference evaluates the convolution with cuFFT on
// reflect-padded tiles (:510-625); here it is evaluated directly, which gives the
// same linear convolution without FFT round-off.
//
// B200 kernel: one CTA computes a 64 x 16 output tile of one channel (grid.z =
// channel). The reflect-extended input tile and the PSF rows (taps padded with zeros
// to a multiple of 16) are staged in shared memory; each thread owns 8 consecutive
// outputs of one row, folds the PSF's vertical symmetry by summing rows y+dy and
// y-dy before the taps, and runs 16-tap chunks out of a register window, so shared
// loads stay near 0.3 per FMA.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "fjb_diffusion.h"
#include "fjb_launches.h"

namespace fjb {

namespace {

constexpr int kTileW = 64;
constexpr int kTileH = 16;
constexpr int kPerThread = 8;
constexpr int kThreads = (kTileW / kPerThread) * kTileH; // 128
constexpr int kChunk = 16;

__device__ __forceinline__ int reflect_whole(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * (n - 1);
    int v = i % period;
    if (v < 0) v += period;
    return v < n ? v : period - v;
}

struct DiffusionPass {
    int width, height, radius, taps; // taps = (2r+1) rounded up to a multiple of 16
    float fraction;
    const float* psf[3]; // per channel, (r+1) rows x taps: row dy holds w(|dy|, dx), dx = -r..r, zero padded
    float* planes[3];    // outputs (never the inputs)
    const float* src[3];
    long long stride;
};

__global__ void __launch_bounds__(kThreads) diffusion_kernel(const __grid_constant__ DiffusionPass P) {
    extern __shared__ float smem[];
    const int r = P.radius;
    const int T = P.taps;
    const int tileCols = kTileW + T - 1;
    const int tileRows = kTileH + 2 * r;
    float* tile = smem;                            // tileRows x tileCols
    float* w = smem + (size_t)tileRows * tileCols; // (r+1) x T
    const int ch = blockIdx.z;
    const float* in = P.src[ch];
    const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH;
    for (int i = threadIdx.x; i < tileRows * tileCols; i += kThreads) {
        const int ty = i / tileCols, tx = i - ty * tileCols;
        const int sy = reflect_whole(y0 - r + ty, P.height);
        const int sx = reflect_whole(x0 - r + tx, P.width);
        tile[i] = in[(long long)sy * P.stride + sx];
    }
    for (int i = threadIdx.x; i < (r + 1) * T; i += kThreads) w[i] = P.psf[ch][i];
    __syncthreads();

    const int lx = (threadIdx.x % (kTileW / kPerThread)) * kPerThread;
    const int ly = threadIdx.x / (kTileW / kPerThread);
    float acc[kPerThread];
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) acc[k] = 0.0f;
    for (int dy = 0; dy <= r; ++dy) {
        const float* rowA = tile + (size_t)(ly + r + dy) * tileCols + lx;
        const float* rowB = tile + (size_t)(ly + r - dy) * tileCols + lx;
        const float* wr = w + (size_t)dy * T;
        for (int c = 0; c < T; c += kChunk) {
            float win[kPerThread + kChunk - 1];
            if (dy == 0) {
#pragma unroll
                for (int j = 0; j < kPerThread + kChunk - 1; ++j) win[j] = rowA[c + j];
            } else {
#pragma unroll
                for (int j = 0; j < kPerThread + kChunk - 1; ++j) win[j] = rowA[c + j] + rowB[c + j];
            }
#pragma unroll
            for (int j = 0; j < kChunk; ++j) {
                const float wj = wr[c + j];
#pragma unroll
                for (int k = 0; k < kPerThread; ++k) acc[k] = fmaf(wj, win[k + j], acc[k]);
            }
        }
    }
    const int y = y0 + ly;
    if (y >= P.height) return;
    float* out = P.planes[ch] + (long long)y * P.stride;
    const float f = P.fraction;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const int x = x0 + lx + k;
        if (x < P.width) {
            const float cur = tile[(size_t)(ly + r) * tileCols + lx + k + r];
            out[x] = (1.0f - f) * cur + f * acc[k];
        }
    }
}

} // namespace

bool diffusion_psf_rows(const double lambda_px[9], const double weights[9], int radius, std::vector<float>& rows,
                        int& taps, std::string& why) {
    if (radius < 0 || radius > kMaxDiffusionRadius) {
        why = "diffusion radius out of range";
        return false;
    }
    const int d = 2 * radius + 1;
    std::vector<float> grid((size_t)d * d);
    double sum = 0.0;
    const double kTwoPi = 6.283185307179586476925286766559;
    for (int iy = 0; iy < d; ++iy)
        for (int ix = 0; ix < d; ++ix) {
            const int dx = ix - radius, dy = iy - radius;
            const double rho = std::sqrt((double)dx * (double)dx + (double)dy * (double)dy);
            double v = 0.0;
            for (int k = 0; k < 9; ++k) {
                const double l = lambda_px[k];
                v += weights[k] * std::exp(-rho / l) / (kTwoPi * l * l);
            }
            const float stored = (float)v;
            grid[(size_t)iy * d + ix] = stored;
            sum += (double)stored;
        }
    if (!(std::isfinite(sum) && sum > 0.0)) {
        why = "diffusion PSF does not normalise";
        return false;
    }
    taps = ((d + 15) / 16) * 16;
    rows.assign((size_t)(radius + 1) * taps, 0.0f);
    for (int dy = 0; dy <= radius; ++dy)
        for (int ix = 0; ix < d; ++ix)
            rows[(size_t)dy * taps + ix] = (float)((double)grid[(size_t)(dy + radius) * d + ix] / sum);
    return true;
}

size_t diffusion_smem_bytes(int radius) {
    const int d = 2 * radius + 1;
    const int taps = ((d + 15) / 16) * 16;
    return ((size_t)(kTileH + 2 * radius) * (kTileW + taps - 1) + (size_t)(radius + 1) * taps) * sizeof(float);
}

cudaError_t launch_diffusion(const float* const psf_rows[3], int radius, int taps, float fraction, float* dst[3],
                             const float* src[3], long long stride, int width, int height, cudaStream_t stream) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    DiffusionPass P{};
    P.width = width;
    P.height = height;
    P.radius = radius;
    P.taps = taps;
    P.fraction = fraction;
    P.stride = stride;
    for (int c = 0; c < 3; ++c) {
        P.psf[c] = psf_rows[c];
        P.planes[c] = dst[c];
        P.src[c] = src[c];
    }
    const size_t smem = diffusion_smem_bytes(radius);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(diffusion_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((width + kTileW - 1) / kTileW, (height + kTileH - 1) / kTileH, 3);
    fjb::count_launch();
    diffusion_kernel<<<grid, kThreads, smem, stream>>>(P);
    return cudaGetLastError();
}

} // namespace fjb
