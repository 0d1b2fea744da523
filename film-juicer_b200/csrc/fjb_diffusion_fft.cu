// fjb_diffusion_fft.cu -- diffusion (a17) as an FFT convolution, for large radii.
//
// Same result as the direct kernel of fjb_diffusion.cu up to FP32 round-off: the
// reflect-extended frame (whole-sample reflection, r samples on every side) is
// convolved circularly with the PSF on an nx x ny grid (nx >= W + 2r a power of two,
// ny >= H + 2r the shortest of 2^a, 3 2^a and 9 2^a), which equals the linear
// convolution on the W x H interior. The
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
// Transforms: radix-8 Stockham stages (after one radix-2 or radix-4 stage for the
// remainder, and before one or two radix-3 stages when the column length is 3 2^a or
// 9 2^a) in shared memory, natural order in and out. Each thread keeps the values of its
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
constexpr int kC2rPairs = kFftMaxValues / 2; // (k, m - k) pairs a thread holds in the inverse split

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

// Shared-memory position of element i of a line: an XOR swizzle inside aligned groups
// of 16 complex values, which spreads the strided Stockham writes over the banks.
__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 4) & 15); }
// The same for a line of n + 1 entries (n a power of two): the extra entry n keeps its place.
__device__ __forceinline__ int swz_n1(int i, int n) { return i < n ? swz(i) : i; }

// Stages the first `n` entries of exp(-2 pi i k / n) from the global table (ntw entries)
// into shared memory. Caller synchronises after.
__device__ __forceinline__ void stage_twiddles(float2* dst, const float2* tw, int log2n, int log2ntw) {
    const int n = 1 << log2n, shift = log2ntw - log2n;
    for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = tw[(size_t)k << shift];
}

// Twiddle table tw[k] = exp(-2 pi i k / n), k < n.
__global__ void twiddle_kernel(float2* tw, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double s, c;
    sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
}

// Size-R DFT in registers (R = 2, 3, 4, 8); kInverse uses the conjugate roots.
template <int R, bool kInverse>
__device__ __forceinline__ void dft(float2 (&v)[R]) {
    auto add = [](float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); };
    auto sub = [](float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); };
    // multiply by -i (forward) or +i (inverse)
    auto rot = [](float2 a) { return kInverse ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); };
    if constexpr (R == 3) {
        // w = exp(-+2 pi i / 3) = -1/2 -+ i sqrt(3)/2:  X1 = v0 - (v1 + v2)/2 -+ i (sqrt(3)/2)(v1 - v2),
        // X2 = the same with the sign of the last term flipped
        constexpr float s3 = 0.86602540378443864676f; // sqrt(3) / 2
        const float2 t1 = add(v[1], v[2]);
        const float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
        const float2 d = sub(v[1], v[2]);
        const float2 sd = rot(make_float2(s3 * d.x, s3 * d.y));
        v[0] = add(v[0], t1);
        v[1] = add(t2, sd);
        v[2] = sub(t2, sd);
    } else if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = add(a, b);
        v[1] = sub(a, b);
    } else if constexpr (R == 4) {
        const float2 a = add(v[0], v[2]), b = sub(v[0], v[2]);
        const float2 c = add(v[1], v[3]), d = rot(sub(v[1], v[3]));
        v[0] = add(a, c);
        v[1] = add(b, d);
        v[2] = sub(a, c);
        v[3] = sub(b, d);
    } else {
        // even / odd halves, each a size-4 DFT, then the W8^k combination
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        dft<4, kInverse>(e);
        dft<4, kInverse>(o);
        constexpr float h = 0.70710678118654752440f;
        const float2 o1 = kInverse ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                                   : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
        const float2 o2 = rot(o[2]);
        const float2 o3 = kInverse ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                                   : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
        v[0] = add(e[0], o[0]);
        v[4] = sub(e[0], o[0]);
        v[1] = add(e[1], o1);
        v[5] = sub(e[1], o1);
        v[2] = add(e[2], o2);
        v[6] = sub(e[2], o2);
        v[3] = add(e[3], o3);
        v[7] = sub(e[3], o3);
    }
}

// One Stockham stage of radix R over `count` lines of length n = 2^log2n (line
// stride `ls`) already in shared memory, Ns = 2^log2ns. Butterfly j of a line takes
// elements j + r n/R, applies the twiddles w^r with w = exp(-+2 pi i (j mod Ns) /
// (Ns R)) (w, w^2 and w^4 from the table, the other powers by products), a size-R
// DFT, and writes elements (j - j mod Ns) R + j mod Ns + r Ns.
template <int R, bool kInverse>
__device__ __forceinline__ void fft_stage(float2* data, int log2n, int ls, int count, int log2ns, const float2* tw,
                                          int tw_shift) {
    constexpr int kMaxB = kFftMaxValues / R;
    constexpr int kLog2R = R == 2 ? 1 : (R == 4 ? 2 : 3);
    const int log2nb = log2n - kLog2R;
    const int nb = 1 << log2nb;
    const int Ns = 1 << log2ns;
    const int total = count << log2nb;
    const int step_shift = log2n - log2ns - kLog2R + tw_shift; // twiddle index step n / (Ns R), in table units
    float2 v[kMaxB][R];
#pragma unroll
    for (int i = 0; i < kMaxB; ++i) {
        const int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            const int line = b >> log2nb, j = b & (nb - 1);
            const float2* d = data + (size_t)line * ls;
            const int jm = j & (Ns - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) v[i][r] = d[swz(j + r * nb)];
            if (jm != 0) {
                auto fetch = [&](int k) {
                    float2 w = tw[(k * jm) << step_shift];
                    if (kInverse) w.y = -w.y;
                    return w;
                };
                float2 w[R];
                w[1] = fetch(1);
                if constexpr (R >= 4) {
                    w[2] = fetch(2);
                    w[3] = cmul(w[1], w[2]);
                }
                if constexpr (R == 8) {
                    w[4] = fetch(4);
                    w[5] = cmul(w[1], w[4]);
                    w[6] = cmul(w[2], w[4]);
                    w[7] = cmul(w[3], w[4]);
                }
#pragma unroll
                for (int r = 1; r < R; ++r) v[i][r] = cmul(v[i][r], w[r]);
            }
            dft<R, kInverse>(v[i]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kMaxB; ++i) {
        const int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            const int line = b >> log2nb, j = b & (nb - 1);
            float2* d = data + (size_t)line * ls;
            const int jm = j & (Ns - 1);
            const int base = ((j - jm) << kLog2R) + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) d[swz(base + r * Ns)] = v[i][r];
        }
    }
    __syncthreads();
}

// Unnormalised DFT (kInverse: conjugate twiddles) of `count` lines of length n = 2^log2n
// in shared memory: radix-8 stages, after one radix-2 or radix-4 stage for the
// remainder of log2n / 3. Caller synchronises before; ends with a barrier.
template <bool kInverse>
__device__ void fft_lines(float2* data, int n, int log2n, int ls, int count, const float2* tw, int log2tw) {
    const int tw_shift = log2tw - log2n;
    int log2ns = 0;
    if (log2n % 3 == 1) {
        fft_stage<2, kInverse>(data, log2n, ls, count, log2ns, tw, tw_shift);
        log2ns = 1;
    } else if (log2n % 3 == 2) {
        fft_stage<4, kInverse>(data, log2n, ls, count, log2ns, tw, tw_shift);
        log2ns = 2;
    }
    for (; log2ns < log2n; log2ns += 3) fft_stage<8, kInverse>(data, log2n, ls, count, log2ns, tw, tw_shift);
}

// One Stockham stage of radix R (2, 3, 4 or 8) over `count` lines of any length n that
// the stages' radices multiply to (line stride `ls`), Ns the product of the earlier
// stages' radices; tw holds exp(-2 pi i k / n), k < n. The same butterflies as
// fft_stage, with integer index arithmetic in place of shifts and masks.
template <int R, bool kInverse>
__device__ __forceinline__ void fft_stage_g(float2* data, int n, int ls, int count, int Ns, const float2* tw) {
    constexpr int kMaxB = (kFftMaxValues - kFftMaxValues % R) / R;
    const int nb = n / R;
    const int total = count * nb;
    const int step = n / (Ns * R); // twiddle index step n / (Ns R)
    float2 v[kMaxB][R];
#pragma unroll
    for (int i = 0; i < kMaxB; ++i) {
        const int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            const int line = b / nb, j = b - line * nb;
            const float2* d = data + (size_t)line * ls;
            const int jm = j % Ns;
#pragma unroll
            for (int r = 0; r < R; ++r) v[i][r] = d[swz(j + r * nb)];
            if (jm != 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    float2 w = tw[r * jm * step];
                    if (kInverse) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            dft<R, kInverse>(v[i]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kMaxB; ++i) {
        const int b = threadIdx.x + i * blockDim.x;
        if (b < total) {
            const int line = b / nb, j = b - line * nb;
            float2* d = data + (size_t)line * ls;
            const int jm = j % Ns;
            const int base = (j - jm) * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) d[swz(base + r * Ns)] = v[i][r];
        }
    }
    __syncthreads();
}

// Unnormalised DFT of `count` lines of length n = 2^a 3^n3 (n3 <= 2): the power-of-two
// stages as in fft_lines (one radix-2 or radix-4 stage, then radix 8), then n3 radix-3
// stages. Caller synchronises before; ends with a barrier.
template <bool kInverse>
__device__ void fft_lines_g(float2* data, int n, int n3, int ls, int count, const float2* tw) {
    int p2 = n;
    for (int k = 0; k < n3; ++k) p2 /= 3;
    int a = 0;
    while ((1 << a) < p2) ++a;
    int Ns = 1;
    if (a % 3 == 1) {
        fft_stage_g<2, kInverse>(data, n, ls, count, Ns, tw);
        Ns = 2;
    } else if (a % 3 == 2) {
        fft_stage_g<4, kInverse>(data, n, ls, count, Ns, tw);
        Ns = 4;
    }
    for (; Ns < p2; Ns *= 8) fft_stage_g<8, kInverse>(data, n, ls, count, Ns, tw);
    for (int k = 0; k < n3; ++k, Ns *= 3) fft_stage_g<3, kInverse>(data, n, ls, count, Ns, tw);
}

struct FftPass {
    DiffusionFftPlan p;
    const float2* tw;    // row twiddle table, p.ntw entries
    const float2* twc;   // column twiddle table exp(-2 pi i k / ny), p.ny entries
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
    float2* tws = fsm + (size_t)p.rows_per_cta * (m + 1); // exp(-2 pi i k / nx), k < nx
    stage_twiddles(tws, F.tw, p.log2m + 1, p.log2ntw);
    // load: complex sample n of line l = (e[2n], e[2n+1]) of the extended row
    #pragma unroll 8
    for (int i = threadIdx.x; i < L * m; i += blockDim.x) {
        const int l = i >> p.log2m, n = i & (m - 1);
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
        fsm[(size_t)l * m + swz(n)] = make_float2(e[0], e[1]);
    }
    __syncthreads();
    fft_lines<false>(fsm, m, p.log2m, m, L, tws, p.log2m + 1);
    // split into the real transform's bins k = 0..m, written transposed
    float2* out = F.work[ch];
    const int lg = p.log2_rows_per_cta;
    for (int i = threadIdx.x; i < (m + 1) << lg; i += blockDim.x) {
        const int k = i >> lg, l = i & ((1 << lg) - 1);
        if (l >= L) continue;
        const float2* z = fsm + (size_t)l * m;
        const float2 zk = z[swz(k == m ? 0 : k)];
        const float2 zr = z[swz(k == 0 ? 0 : m - k)];
        const float2 zc = make_float2(zr.x, -zr.y);
        const float2 E = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
        const float2 D = make_float2(zk.x - zc.x, zk.y - zc.y);
        const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
        const float2 w = tws[k];
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
    float2* tws = fsm + (size_t)p.cols_per_cta * ny; // exp(-2 pi i k / ny), k < ny
    for (int k = threadIdx.x; k < ny; k += blockDim.x) tws[k] = F.twc[k];
    for (int c = 0; c < KC; ++c) {
        #pragma unroll 4
        for (int ey = threadIdx.x; ey < ny; ey += blockDim.x) {
            float2 v = make_float2(0.0f, 0.0f);
            if (kBuild) {
                // compact PSF row j holds dy = j - r, placed at dy mod ny
                const int dy = ey <= r ? ey : ey - ny;
                if (dy >= -r && dy <= r) v = in[(size_t)(k0 + c) * p.sy + dy + r];
            } else if (ey < rows) {
                v = in[(size_t)(k0 + c) * p.sy + ey];
            }
            fsm[(size_t)c * ny + swz(ey)] = v;
        }
    }
    __syncthreads();
    if (p.ny3 == 0)
        fft_lines<false>(fsm, ny, p.log2ny, ny, KC, tws, p.log2ny);
    else
        fft_lines_g<false>(fsm, ny, p.ny3, ny, KC, tws);
    float* spec = F.spectrum[ch];
    if constexpr (kBuild) {
        const float scale = 1.0f / ((float)p.m * (float)ny);
        for (int c = 0; c < KC; ++c)
            for (int ky = threadIdx.x; ky < ny; ky += blockDim.x)
                spec[(size_t)(k0 + c) * ny + ky] = fsm[(size_t)c * ny + swz(ky)].x * scale;
        return;
    }
    for (int c = 0; c < KC; ++c) {
        #pragma unroll 4
        for (int ky = threadIdx.x; ky < ny; ky += blockDim.x) {
            const float s = spec[(size_t)(k0 + c) * ny + ky];
            float2& v = fsm[(size_t)c * ny + swz(ky)];
            v = make_float2(v.x * s, v.y * s);
        }
    }
    __syncthreads();
    if (p.ny3 == 0)
        fft_lines<true>(fsm, ny, p.log2ny, ny, KC, tws, p.log2ny);
    else
        fft_lines_g<true>(fsm, ny, p.ny3, ny, KC, tws);
    float2* out = F.work[ch];
    const int H = p.height;
    for (int c = 0; c < KC; ++c)
        for (int y = threadIdx.x; y < H; y += blockDim.x) out[(size_t)(k0 + c) * p.sy + r + y] = fsm[(size_t)c * ny + swz(r + y)];
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
    float2* tws = fsm + (size_t)p.rows_per_cta * ls; // exp(-2 pi i k / nx), k < nx
    stage_twiddles(tws, F.tw, p.log2m + 1, p.log2ntw);
    const int lg = p.log2_rows_per_cta;
    #pragma unroll 8
    for (int i = threadIdx.x; i < (m + 1) << lg; i += blockDim.x) {
        const int k = i >> lg, l = i & ((1 << lg) - 1);
        if (l < L) fsm[(size_t)l * ls + swz_n1(k, m)] = in[(size_t)k * p.sy + r + y0 + l];
    }
    __syncthreads();
    // Z[k] = E[k] + i O[k], E = (X[k] + conj X[m-k]) / 2, O = (X[k] - conj X[m-k]) conj(w^k) / 2.
    // A thread takes pairs (k, m - k), 0 <= k < m/2, reads both bins, and writes Z[k] and
    // Z[m - k] (k > 0) after the barrier; the middle bin m/2 of line l goes to thread l.
    const int half = m / 2, log2half = p.log2m - 1;
    constexpr int kMaxPairs = kC2rPairs;
    float2 zk[kMaxPairs], zm[kMaxPairs];
    auto z_of = [&](float2 xk, float2 xm, int k) {
        const float2 xc = make_float2(xm.x, -xm.y);
        const float2 E = make_float2(0.5f * (xk.x + xc.x), 0.5f * (xk.y + xc.y));
        const float2 D = make_float2(0.5f * (xk.x - xc.x), 0.5f * (xk.y - xc.y));
        const float2 w = tws[k];
        const float2 O = cmul(D, make_float2(w.x, -w.y));
        return make_float2(E.x - O.y, E.y + O.x);
    };
#pragma unroll
    for (int q = 0; q < kMaxPairs; ++q) {
        const int i = threadIdx.x + q * blockDim.x;
        if (i < L << log2half) {
            const int l = i >> log2half, k = i & (half - 1);
            const float2* x = fsm + (size_t)l * ls;
            const float2 a = x[swz(k)], b = x[swz_n1(m - k, m)];
            zk[q] = z_of(a, b, k);
            zm[q] = z_of(b, a, m - k);
        }
    }
    float2 zmid = make_float2(0.0f, 0.0f);
    if ((int)threadIdx.x < L) {
        const float2 a = fsm[(size_t)threadIdx.x * ls + swz(half)];
        zmid = z_of(a, a, half);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kMaxPairs; ++q) {
        const int i = threadIdx.x + q * blockDim.x;
        if (i < L << log2half) {
            const int l = i >> log2half, k = i & (half - 1);
            float2* x = fsm + (size_t)l * ls;
            x[swz(k)] = zk[q];
            if (k > 0) x[swz(m - k)] = zm[q]; // 0 < k: m - k < m
        }
    }
    if ((int)threadIdx.x < L) fsm[(size_t)threadIdx.x * ls + swz(half)] = zmid;
    __syncthreads();
    fft_lines<true>(fsm, m, p.log2m, ls, L, tws, p.log2m + 1);
    const float f = F.fraction;
    for (int l = 0; l < L; ++l)
        #pragma unroll 4
        for (int x = threadIdx.x; x < W; x += blockDim.x) {
            const int ex = x + r;
            const float2 z = fsm[(size_t)l * ls + swz(ex >> 1)];
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

// data lines, then the twiddle table of the transform length
size_t rows_smem(const DiffusionFftPlan& p) {
    return ((size_t)p.rows_per_cta * (p.m + 1) + 2 * (size_t)p.m) * sizeof(float2);
}
size_t cols_smem(const DiffusionFftPlan& p) { return ((size_t)p.cols_per_cta + 1) * p.ny * sizeof(float2); }

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
    // columns: the shortest 2^a, 3 2^a or 9 2^a (a >= 4, at most kFftMaxLen) holding the
    // extended rows
    int ny = 0, ny3 = 0;
    for (int k = 0, f = 1; k <= 2; ++k, f *= 3) {
        long long n = 16LL * f;
        while (n < hy) n *= 2;
        if (n <= kFftMaxLen && (ny == 0 || n < ny)) {
            ny = (int)n;
            ny3 = k;
        }
    }
    if (ny == 0) return false;
    p.width = width;
    p.height = height;
    p.radius = radius;
    p.m = nx / 2;
    p.log2m = log2_exact(p.m);
    p.ny = ny;
    p.ny3 = ny3;
    p.log2ny = ny3 == 0 ? log2_exact(ny) : -1;
    p.ntw = nx;
    p.log2ntw = log2_exact(p.ntw);
    p.ey = height + 2 * radius;
    p.sy = (p.ey + 3) / 4 * 4;
    // every thread holds at most kFftMaxValues values of a stage
    p.rows_per_cta = (kFftThreads * kFftMaxValues) / p.m;
    if (p.rows_per_cta > 4) p.rows_per_cta = 4;
    // a radix-3 stage holds 5 butterflies (15 values) per thread
    p.cols_per_cta = (kFftThreads * (ny3 ? kFftMaxValues - kFftMaxValues % 3 : kFftMaxValues)) / ny;
    if (p.cols_per_cta > 4) p.cols_per_cta = 4;
    if (p.rows_per_cta < 1 || p.cols_per_cta < 1) return false;
    // the inverse split holds 2 values per (k, m - k) pair: (m/2 + 1) pairs per row
    if ((long long)p.rows_per_cta * (p.m / 2) > (long long)kFftThreads * kC2rPairs) return false;
    p.log2_rows_per_cta = log2_exact(p.rows_per_cta);
    p.work_floats = (size_t)3 * (p.m + 1) * p.sy * 2;
    p.spectrum_floats = (size_t)2 * p.ntw + (size_t)2 * ny + (size_t)3 * (p.m + 1) * ny;
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
    F.twc = tw + p.ntw;
    for (int c = 0; c < 3; ++c) {
        F.spectrum[c] = spectrum + (size_t)2 * (p.ntw + p.ny) + (size_t)c * (p.m + 1) * p.ny;
        F.work[c] = reinterpret_cast<float2*>(work) + (size_t)c * (p.m + 1) * p.sy;
        F.psf[c] = psf_rows[c];
    }
    F.taps = taps;
    cudaError_t e;
    fjb::count_launch();
    twiddle_kernel<<<(p.ntw + 255) / 256, 256, 0, stream>>>(tw, p.ntw);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    fjb::count_launch();
    twiddle_kernel<<<(p.ny + 255) / 256, 256, 0, stream>>>(tw + p.ntw, p.ny);
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
    F.twc = F.tw + p.ntw;
    for (int c = 0; c < 3; ++c) {
        F.spectrum[c] = const_cast<float*>(spectrum) + (size_t)2 * (p.ntw + p.ny) + (size_t)c * (p.m + 1) * p.ny;
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
