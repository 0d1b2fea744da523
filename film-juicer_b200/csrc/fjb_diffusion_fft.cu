// fjb_diffusion_fft.cu -- diffusion (a17) as an FFT convolution, for large radii.
//
// Same result as the direct kernel of fjb_diffusion.cu up to FP32 round-off: the
// reflect-extended frame (whole-sample reflection, r samples on every side) is
// convolved circularly with the PSF on an nx x ny grid (powers of two, nx >= W + 2r,
// ny >= H + 2r), which equals the linear convolution on the W x H interior. The
// reference reaches the same convolution with cuFFT on reflect-padded tiles
// (src/Cuda/Diffusion/JuicerCudaDiffusion.cu:510-625); the transforms here are written
// in this file.
//
// Schedule per frame (all three channels in each launch, grid.z / grid.y = channel):
//   rows_r2c   : L extended rows per CTA; each row is a real sequence of nx samples,
//                transformed as nx/2 complex points plus the even/odd split, and
//                written transposed (spectrum column k, row ey) so that the column
//                pass reads contiguous columns;
//   columns    : KC spectrum columns per CTA: forward FFT over ny, multiply by the
//                PSF spectrum (real: the PSF is even in both axes; scaled by
//                1 / (nx/2 * ny) to fold in the inverse normalisation), inverse FFT,
//                and only the rows the output needs are written back;
//   rows_c2r   : L output rows per CTA: inverse of the even/odd split, inverse FFT,
//                crop to the interior and mix (1 - f) x + f (PSF * x).
// The PSF spectrum is built once per descriptor and frame size by the same row and
// column transforms over the PSF placed around the origin.
//
// Transforms: radix-4 Stockham stages (one radix-2 stage first when log2 n is odd)
// in shared memory, natural order in and out. Each thread keeps the values of its
// butterflies in registers across the stage barrier, so one buffer per line is
// enough. Twiddles come from a table exp(-2 pi i k / N) built in FP64 and rounded.
#include <cuda_runtime.h>

#include "fjb_diffusion.h"
#include "fjb_launches.h"

namespace fjb {

namespace {

constexpr int kFftThreads = 512;
constexpr int kFftMaxValues = 16; // complex values a thread holds across a stage barrier
constexpr int kFftMaxLen = 8192;  // longest transform (nx / 2 and ny)
constexpr int kC2rPairs = kFftMaxValues / 2 + 1; // (k, m - k) pairs a thread holds in the inverse split

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ int reflect_whole(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * (n - 1);
    int v = i % period;
    if (v < 0) v += period;
    return v < n ? v : period - v;
}

// Twiddle table tw[k] = exp(-2 pi i k / n), k < n.
__global__ void twiddle_kernel(float2* tw, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double s, c;
    sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
}

// One Stockham stage of radix R over `count` lines of length n (line stride `ls`)
// already in shared memory. Butterfly b of a line takes elements j + r n/R, applies
// the twiddles exp(-+2 pi i r (j mod Ns) / (Ns R)), a size-R DFT, and writes elements
// (j - j mod Ns) R + j mod Ns + r Ns.
template <int R, bool kInverse>
__device__ __forceinline__ void fft_stage(float2* data, int n, int ls, int count, int Ns, const float2* tw,
                                          int tw_shift) {
    constexpr int kMaxB = kFftMaxValues / R;
    const int nb = n / R;
    const int total = count * nb;
    const int step = n / (Ns * R); // twiddle index step, in units of 2 pi / n
    float2 v[kMaxB][R];
#pragma unroll
    for (int i = 0; i < kMaxB; ++i) {
        const int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            const int line = b / nb, j = b - line * nb;
            const float2* d = data + (size_t)line * ls;
            const int jm = j & (Ns - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                float2 x = d[j + r * nb];
                if (r > 0) {
                    float2 w = tw[(r * jm * step) << tw_shift];
                    if (kInverse) w.y = -w.y;
                    x = cmul(x, w);
                }
                v[i][r] = x;
            }
            if (R == 2) {
                const float2 a = v[i][0], b2 = v[i][1];
                v[i][0] = make_float2(a.x + b2.x, a.y + b2.y);
                v[i][1] = make_float2(a.x - b2.x, a.y - b2.y);
            } else {
                const float2 a = make_float2(v[i][0].x + v[i][2].x, v[i][0].y + v[i][2].y);
                const float2 bb = make_float2(v[i][0].x - v[i][2].x, v[i][0].y - v[i][2].y);
                const float2 c = make_float2(v[i][1].x + v[i][3].x, v[i][1].y + v[i][3].y);
                const float2 dd = make_float2(v[i][1].x - v[i][3].x, v[i][1].y - v[i][3].y);
                // forward: -i d; inverse: +i d
                const float2 md = kInverse ? make_float2(-dd.y, dd.x) : make_float2(dd.y, -dd.x);
                v[i][0] = make_float2(a.x + c.x, a.y + c.y);
                v[i][1] = make_float2(bb.x + md.x, bb.y + md.y);
                v[i][2] = make_float2(a.x - c.x, a.y - c.y);
                v[i][3] = make_float2(bb.x - md.x, bb.y - md.y);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kMaxB; ++i) {
        const int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            const int line = b / nb, j = b - line * nb;
            float2* d = data + (size_t)line * ls;
            const int jm = j & (Ns - 1);
            const int base = (j - jm) * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) d[base + r * Ns] = v[i][r];
        }
    }
    __syncthreads();
}

// Unnormalised DFT (kInverse: conjugate twiddles) of `count` lines of length n = 2^log2n
// in shared memory. Caller synchronises before; ends with a barrier.
template <bool kInverse>
__device__ void fft_lines(float2* data, int n, int log2n, int ls, int count, const float2* tw, int log2tw) {
    const int tw_shift = log2tw - log2n;
    int Ns = 1;
    if (log2n & 1) {
        fft_stage<2, kInverse>(data, n, ls, count, Ns, tw, tw_shift);
        Ns = 2;
    }
    for (; Ns < n; Ns *= 4) fft_stage<4, kInverse>(data, n, ls, count, Ns, tw, tw_shift);
}

struct FftPass {
    DiffusionFftPlan p;
    const float2* tw;    // twiddle table, p.ntw entries
    float2* work[3];     // per channel: (m + 1) columns x sy rows (transposed spectrum)
    float* spectrum[3];  // per channel: (m + 1) x ny reals, scaled
    const float* src[3]; // frame planes (apply) or unused (spectrum build)
    float* dst[3];
    long long stride;
    const float* psf[3]; // PSF rows |dy| = 0..r, taps each (spectrum build)
    int taps;
    float fraction;
};

// Row forward transforms. kPsf: the rows of the PSF placed around the origin
// (compact row i holds dy = i - r); otherwise the reflect-extended frame rows.
template <bool kPsf>
__global__ void __launch_bounds__(kFftThreads) rows_r2c_kernel(const __grid_constant__ FftPass F) {
    extern __shared__ float2 fsm[];
    const DiffusionFftPlan& p = F.p;
    const int ch = blockIdx.y;
    const int m = p.m, nx = 2 * m, r = p.radius;
    const int rows = kPsf ? 2 * r + 1 : p.ey;
    const int row0 = blockIdx.x * p.rows_per_cta;
    const int L = min(p.rows_per_cta, rows - row0);
    if (L <= 0) return;
    const int W = p.width, H = p.height;
    // load: complex sample n of line l = (e[2n], e[2n+1]) of the extended row
    for (int i = threadIdx.x; i < L * m; i += blockDim.x) {
        const int l = i / m, n = i - l * m;
        const int ey = row0 + l;
        float e[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int ex = 2 * n + h;
            float v = 0.0f;
            if (kPsf) {
                const int dy = ey - r;
                const int dx = ex <= r ? ex : ex - nx; // circular placement
                if (dx >= -r && dx <= r) v = F.psf[ch][(size_t)(dy < 0 ? -dy : dy) * F.taps + dx + r];
            } else if (ex < W + 2 * r) {
                const int yy = ey - r, xx = ex - r;
                const int sy = (unsigned)yy < (unsigned)H ? yy : reflect_whole(yy, H);
                const int sx = (unsigned)xx < (unsigned)W ? xx : reflect_whole(xx, W);
                v = F.src[ch][(long long)sy * F.stride + sx];
            }
            e[h] = v;
        }
        fsm[(size_t)l * m + n] = make_float2(e[0], e[1]);
    }
    __syncthreads();
    fft_lines<false>(fsm, m, p.log2m, m, L, F.tw, p.log2ntw);
    // split into the real transform's bins k = 0..m, written transposed
    float2* out = F.work[ch];
    const int shift_nx = p.log2ntw - (p.log2m + 1);
    for (int i = threadIdx.x; i < L * (m + 1); i += blockDim.x) {
        const int k = i / L, l = i - k * L;
        const float2* z = fsm + (size_t)l * m;
        const float2 zk = z[k == m ? 0 : k];
        const float2 zr = z[k == 0 ? 0 : m - k];
        const float2 zc = make_float2(zr.x, -zr.y);
        const float2 E = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
        const float2 D = make_float2(zk.x - zc.x, zk.y - zc.y);
        const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
        const float2 w = F.tw[(size_t)k << shift_nx];
        const float2 wo = cmul(w, O);
        out[(size_t)k * p.sy + row0 + l] = make_float2(E.x + wo.x, E.y + wo.y);
    }
}

// Spectrum columns. kBuild: forward transform of the PSF rows and keep the scaled real
// part; otherwise forward transform, multiply by the PSF spectrum, inverse transform,
// and write back the rows [r, r + H) the output needs.
template <bool kBuild>
__global__ void __launch_bounds__(kFftThreads) columns_kernel(const __grid_constant__ FftPass F) {
    extern __shared__ float2 fsm[];
    const DiffusionFftPlan& p = F.p;
    const int ch = blockIdx.y;
    const int ny = p.ny, r = p.radius;
    const int k0 = blockIdx.x * p.cols_per_cta;
    const int KC = min(p.cols_per_cta, p.m + 1 - k0);
    if (KC <= 0) return;
    const float2* in = F.work[ch];
    const int rows = kBuild ? 2 * r + 1 : p.ey;
    for (int i = threadIdx.x; i < KC * ny; i += blockDim.x) {
        const int c = i / ny, ey = i - c * ny;
        float2 v = make_float2(0.0f, 0.0f);
        if (kBuild) {
            // compact PSF row j holds dy = j - r, placed at dy mod ny
            const int dy = ey <= r ? ey : ey - ny;
            if (dy >= -r && dy <= r) v = in[(size_t)(k0 + c) * p.sy + dy + r];
        } else if (ey < rows) {
            v = in[(size_t)(k0 + c) * p.sy + ey];
        }
        fsm[i] = v;
    }
    __syncthreads();
    fft_lines<false>(fsm, ny, p.log2ny, ny, KC, F.tw, p.log2ntw);
    float* spec = F.spectrum[ch];
    if (kBuild) {
        const float scale = 1.0f / ((float)p.m * (float)ny);
        for (int i = threadIdx.x; i < KC * ny; i += blockDim.x) spec[(size_t)k0 * ny + i] = fsm[i].x * scale;
        return;
    }
    for (int i = threadIdx.x; i < KC * ny; i += blockDim.x) {
        const float s = spec[(size_t)k0 * ny + i];
        fsm[i] = make_float2(fsm[i].x * s, fsm[i].y * s);
    }
    __syncthreads();
    fft_lines<true>(fsm, ny, p.log2ny, ny, KC, F.tw, p.log2ntw);
    float2* out = F.work[ch];
    const int H = p.height;
    for (int i = threadIdx.x; i < KC * H; i += blockDim.x) {
        const int c = i / H, y = i - c * H;
        out[(size_t)(k0 + c) * p.sy + r + y] = fsm[(size_t)c * ny + r + y];
    }
}

// Output rows: inverse real transform of spectrum rows r + y, crop, mix.
__global__ void __launch_bounds__(kFftThreads) rows_c2r_kernel(const __grid_constant__ FftPass F) {
    extern __shared__ float2 fsm[];
    const DiffusionFftPlan& p = F.p;
    const int ch = blockIdx.y;
    const int m = p.m, r = p.radius, W = p.width, H = p.height;
    const int ls = m + 1;
    const int y0 = blockIdx.x * p.rows_per_cta;
    const int L = min(p.rows_per_cta, H - y0);
    if (L <= 0) return;
    const float2* in = F.work[ch];
    for (int i = threadIdx.x; i < L * (m + 1); i += blockDim.x) {
        const int k = i / L, l = i - k * L;
        fsm[(size_t)l * ls + k] = in[(size_t)k * p.sy + r + y0 + l];
    }
    __syncthreads();
    // Z[k] = E[k] + i O[k], E = (X[k] + conj X[m-k]) / 2, O = (X[k] - conj X[m-k]) conj(w^k) / 2;
    // each thread takes the pair (k, m - k), reads both, then writes both after the barrier
    const int shift_nx = p.log2ntw - (p.log2m + 1);
    const int half = m / 2;
    constexpr int kMaxPairs = kC2rPairs;
    float2 zk[kMaxPairs], zm[kMaxPairs];
    auto z_of = [&](float2 xk, float2 xm, int k) {
        const float2 xc = make_float2(xm.x, -xm.y);
        const float2 E = make_float2(0.5f * (xk.x + xc.x), 0.5f * (xk.y + xc.y));
        const float2 D = make_float2(0.5f * (xk.x - xc.x), 0.5f * (xk.y - xc.y));
        const float2 w = F.tw[(size_t)k << shift_nx];
        const float2 O = cmul(D, make_float2(w.x, -w.y));
        return make_float2(E.x - O.y, E.y + O.x);
    };
#pragma unroll
    for (int q = 0; q < kMaxPairs; ++q) {
        const int i = threadIdx.x + q * blockDim.x;
        if (i < L * (half + 1)) {
            const int l = i / (half + 1), k = i - l * (half + 1);
            const float2* x = fsm + (size_t)l * ls;
            const float2 a = x[k], b = x[m - k];
            zk[q] = z_of(a, b, k);
            zm[q] = z_of(b, a, m - k); // used when 0 < k < m/2
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kMaxPairs; ++q) {
        const int i = threadIdx.x + q * blockDim.x;
        if (i < L * (half + 1)) {
            const int l = i / (half + 1), k = i - l * (half + 1);
            float2* x = fsm + (size_t)l * ls;
            x[k] = zk[q];
            if (k > 0 && k < half) x[m - k] = zm[q];
        }
    }
    __syncthreads();
    fft_lines<true>(fsm, m, p.log2m, ls, L, F.tw, p.log2ntw);
    const float f = F.fraction;
    for (int i = threadIdx.x; i < L * W; i += blockDim.x) {
        const int l = i / W, x = i - l * W;
        const int ex = x + r;
        const float2 z = fsm[(size_t)l * ls + (ex >> 1)];
        const float conv = (ex & 1) ? z.y : z.x;
        const long long o = (long long)(y0 + l) * F.stride + x;
        const float cur = F.src[ch][o];
        F.dst[ch][o] = (1.0f - f) * cur + f * conv;
    }
}

int log2_exact(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

int pow2_at_least(int n) { return 1 << log2_exact(n); }

size_t rows_smem(const DiffusionFftPlan& p) { return (size_t)p.rows_per_cta * (p.m + 1) * sizeof(float2); }
size_t cols_smem(const DiffusionFftPlan& p) { return (size_t)p.cols_per_cta * p.ny * sizeof(float2); }

cudaError_t set_smem(const void* fn, size_t bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

} // namespace

bool diffusion_fft_plan(int width, int height, int radius, DiffusionFftPlan& p) {
    p = DiffusionFftPlan{};
    if (width <= 0 || height <= 0 || radius < 0) return false;
    const long long wx = (long long)width + 2LL * radius, hy = (long long)height + 2LL * radius;
    if (wx > 2LL * kFftMaxLen || hy > kFftMaxLen) return false;
    const int nx = pow2_at_least((int)(wx < 16 ? 16 : wx));
    const int ny = pow2_at_least((int)(hy < 16 ? 16 : hy));
    p.width = width;
    p.height = height;
    p.radius = radius;
    p.m = nx / 2;
    p.log2m = log2_exact(p.m);
    p.ny = ny;
    p.log2ny = log2_exact(ny);
    p.ntw = nx > ny ? nx : ny;
    p.log2ntw = log2_exact(p.ntw);
    p.ey = height + 2 * radius;
    p.sy = (p.ey + 3) / 4 * 4;
    // every thread holds at most kFftMaxValues values of a stage
    p.rows_per_cta = (kFftThreads * kFftMaxValues) / p.m;
    if (p.rows_per_cta > 4) p.rows_per_cta = 4;
    p.cols_per_cta = (kFftThreads * kFftMaxValues) / ny;
    if (p.cols_per_cta > 2) p.cols_per_cta = 2;
    if (p.rows_per_cta < 1 || p.cols_per_cta < 1) return false;
    // the inverse split holds 2 values per (k, m - k) pair: (m/2 + 1) pairs per row
    if ((long long)p.rows_per_cta * (p.m / 2 + 1) > (long long)kFftThreads * kC2rPairs) return false;
    p.work_floats = (size_t)3 * (p.m + 1) * p.sy * 2;
    p.spectrum_floats = (size_t)2 * p.ntw + (size_t)3 * (p.m + 1) * ny;
    return true;
}

bool diffusion_prefers_fft(int width, int height, int radius) {
    DiffusionFftPlan p;
    return radius >= kDiffusionFftMinRadius && diffusion_fft_plan(width, height, radius, p);
}

cudaError_t launch_diffusion_fft_spectrum(const DiffusionFftPlan& p, const float* const psf_rows[3], int taps,
                                          float* spectrum, float* work, cudaStream_t stream) {
    FftPass F{};
    F.p = p;
    float2* tw = reinterpret_cast<float2*>(spectrum);
    F.tw = tw;
    for (int c = 0; c < 3; ++c) {
        F.spectrum[c] = spectrum + (size_t)2 * p.ntw + (size_t)c * (p.m + 1) * p.ny;
        F.work[c] = reinterpret_cast<float2*>(work) + (size_t)c * (p.m + 1) * p.sy;
        F.psf[c] = psf_rows[c];
    }
    F.taps = taps;
    cudaError_t e;
    fjb::count_launch();
    twiddle_kernel<<<(p.ntw + 255) / 256, 256, 0, stream>>>(tw, p.ntw);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t rs = rows_smem(p), cs = cols_smem(p);
    if ((e = set_smem((const void*)rows_r2c_kernel<true>, rs)) != cudaSuccess) return e;
    if ((e = set_smem((const void*)columns_kernel<true>, cs)) != cudaSuccess) return e;
    const int psf_rows_n = 2 * p.radius + 1;
    fjb::count_launch();
    rows_r2c_kernel<true><<<dim3((psf_rows_n + p.rows_per_cta - 1) / p.rows_per_cta, 3), kFftThreads, rs, stream>>>(F);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    fjb::count_launch();
    columns_kernel<true><<<dim3((p.m + 1 + p.cols_per_cta - 1) / p.cols_per_cta, 3), kFftThreads, cs, stream>>>(F);
    return cudaGetLastError();
}

cudaError_t launch_diffusion_fft(const DiffusionFftPlan& p, const float* spectrum, float fraction, float* dst[3],
                                 const float* src[3], long long stride, float* work, cudaStream_t stream) {
    FftPass F{};
    F.p = p;
    F.tw = reinterpret_cast<const float2*>(spectrum);
    for (int c = 0; c < 3; ++c) {
        F.spectrum[c] = const_cast<float*>(spectrum) + (size_t)2 * p.ntw + (size_t)c * (p.m + 1) * p.ny;
        F.work[c] = reinterpret_cast<float2*>(work) + (size_t)c * (p.m + 1) * p.sy;
        F.src[c] = src[c];
        F.dst[c] = dst[c];
    }
    F.stride = stride;
    F.fraction = fraction;
    cudaError_t e;
    const size_t rs = rows_smem(p), cs = cols_smem(p);
    if ((e = set_smem((const void*)rows_r2c_kernel<false>, rs)) != cudaSuccess) return e;
    if ((e = set_smem((const void*)columns_kernel<false>, cs)) != cudaSuccess) return e;
    if ((e = set_smem((const void*)rows_c2r_kernel, rs)) != cudaSuccess) return e;
    fjb::count_launch();
    rows_r2c_kernel<false><<<dim3((p.ey + p.rows_per_cta - 1) / p.rows_per_cta, 3), kFftThreads, rs, stream>>>(F);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    fjb::count_launch();
    columns_kernel<false><<<dim3((p.m + 1 + p.cols_per_cta - 1) / p.cols_per_cta, 3), kFftThreads, cs, stream>>>(F);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    fjb::count_launch();
    rows_c2r_kernel<<<dim3((p.height + p.rows_per_cta - 1) / p.rows_per_cta, 3), kFftThreads, rs, stream>>>(F);
    return cudaGetLastError();
}

} // namespace fjb
