// fjb_grain.cu -- density-space visual grain (a15).
//
// Per CMY channel the grain is the sum over up to three particle-size scales (fine,
// mid, coarse) of a correlated delta: a Poisson particle sample per pixel (one
// layer, or the three emulsion sublayers, each optionally blurred by its dye-cloud
// Gaussian) minus the developed density, blurred by the scale's correlation
// Gaussian and weighted; a shared (chroma-correlated) delta may be mixed in; the
// result is added back to the density planes in place.
//
// Arithmetic restates the reference's grain path so that results are bit-identical:
//   random draws     src/Cuda/Film/JuicerCudaFilmPipeline.cu:1892-1995 (static blue
//                    noise lookups keyed by splitmix64 of the draw index, or the
//                    Philox4x32-10 counter stream of third_party/openrand/philox.h)
//   Poisson / model  :1997-2075 (product-of-uniforms below lambda 10, rounded normal
//                    above; saturating particle count)
//   Wang offsets     :1674-1775, value noise / breathing / clump :1777-1890
//   frame uniforms   :2174-2352
//   layer lookup     :2077-2171
//   sample kernels   :2579-2986 (simple, one layer, layer triplet)
//   schedule, blurs  src/Cuda/Scan/JuicerCudaScanPipeline.cu:3141-3740, :317-380,
//                    :454-578, :705-775 (FMA chains in tap order, half-sample
//                    reflection, sanitising stores)
// The float contractions the reference's compiler forms (a + b * c -> fma) are
// written out as explicit __fmaf_rn here so that they do not depend on this
// compiler's choices. The layout is this project's: fewer passes (sample and
// accumulate/delta fused, the gain folded into the last weighted pass, mix and
// reconstruction in one pass) and taps passed as kernel parameters.
#include <cuda_runtime.h>

#include <cstdint>

#include "fjb_grain.h"
#include "fjb_launches.h"
#include "fjb_philox.cuh"

namespace fjb {

namespace {

constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvU32 = 1.0f / 4294967296.0f;

__device__ __forceinline__ bool finite(float v) { return isfinite(v); }
__device__ __forceinline__ float sanitize(float v) { return isfinite(v) ? v : 0.0f; }
__device__ __forceinline__ float clamp01(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

__device__ __forceinline__ uint64_t splitmix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ULL;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}

__device__ __forceinline__ int wrap_coordinate(int64_t c, int size) {
    if (size <= 0) return 0;
    if ((size & (size - 1)) == 0) return (int)((uint64_t)c & (uint64_t)(size - 1));
    c %= (int64_t)size;
    if (c < 0) c += size;
    return (int)c;
}

__device__ __forceinline__ float smoothstep(float t) { return (t * t) * __fmaf_rn(-2.0f, t, 3.0f); }

__device__ __forceinline__ float hash01(int x, int y, uint64_t seed) {
    const uint64_t h = splitmix64(seed ^ ((uint64_t)x * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)y * 0xBF58476D1CE4E5B9ULL));
    return (float)(uint32_t)(h & 0xFFFFFFFFu) * kInvU32;
}

__device__ __forceinline__ float spatial_hash01(int x, int y, uint64_t seed) {
    const uint32_t lo = (uint32_t)seed, hi = (uint32_t)(seed >> 32);
    uint32_t h = lo ^ ((hi << 16) | (hi >> 16));
    h ^= (uint32_t)x * 0x9E3779B9u;
    h ^= (uint32_t)y * 0x85EBCA6Bu;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return (float)h * kInvU32;
}

__device__ __forceinline__ uint32_t hash_u32(int x, int y, uint64_t seed, uint64_t salt) {
    const uint64_t h =
        splitmix64(seed ^ salt ^ ((uint64_t)x * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)y * 0xBF58476D1CE4E5B9ULL));
    return (uint32_t)(h & 0xFFFFFFFFu);
}

__device__ __forceinline__ float value_noise(float cx, float cy, uint64_t seed) {
    const int ix = (int)floorf(cx), iy = (int)floorf(cy);
    const float fx = cx - (float)ix, fy = cy - (float)iy;
    const float sx = smoothstep(fx), sy = smoothstep(fy);
    const float v00 = spatial_hash01(ix, iy, seed);
    const float v10 = spatial_hash01(ix + 1, iy, seed);
    const float v01 = spatial_hash01(ix, iy + 1, seed);
    const float v11 = spatial_hash01(ix + 1, iy + 1, seed);
    const float v0 = __fmaf_rn(v10 - v00, sx, v00);
    const float v1 = __fmaf_rn(v11 - v01, sx, v01);
    return __fmaf_rn(v1 - v0, sy, v0);
}

constexpr uint32_t kPhiloxGlobalSeed = 0xAAAAAAAAu;

struct GrainRng {
    Philox philox;
    const GrainFrame* f;
    uint64_t abs_x, abs_y, seed;
    uint32_t draw;
    int use_stbn, off_x, off_y;
    int64_t pitch_offset;
    size_t frame_row_base;
    const uint8_t* frame_base; // the blue-noise frame's first row
    int mask_w, mask_h;

    __device__ GrainRng(const GrainFrame* frame, uint64_t s, uint64_t ax, uint64_t ay, int stbn, int frame_offset,
                        int wang_x, int wang_y)
        : philox(s, (uint32_t)ax, kPhiloxGlobalSeed, (uint32_t)ay), f(frame), abs_x(ax), abs_y(ay), seed(s),
          draw(0), use_stbn(stbn), off_x(wang_x), off_y(wang_y), pitch_offset(0), frame_row_base(0),
          frame_base(nullptr), mask_w(-1), mask_h(-1) {
        if (!use_stbn) return;
        if ((f->stbn_w & (f->stbn_w - 1)) == 0 && (f->stbn_h & (f->stbn_h - 1)) == 0) {
            mask_w = f->stbn_w - 1;
            mask_h = f->stbn_h - 1;
        }
        if (f->pitch_px > 0) pitch_offset = (int64_t)f->pitch_px * (f->frame_index + (int64_t)frame_offset);
        const int wf = wrap_coordinate((int64_t)f->stbn_frame + (int64_t)frame_offset, f->stbn_frames);
        frame_row_base = (size_t)wf * (size_t)f->stbn_h;
        frame_base = f->stbn + frame_row_base * (size_t)f->stbn_w;
    }

    // The blue-noise uniform of draw d (its table address depends on d alone).
    __device__ __forceinline__ float stbn_at(uint32_t d) const {
        const uint64_t h = splitmix64(seed + (uint64_t)d * 0x9E3779B97F4A7C15ULL);
        const int ox = (int)(h & 0xFFFFu) + off_x;
        const int oy = (int)((h >> 16) & 0xFFFFu) + off_y;
        if (mask_w >= 0) {
            // power-of-two table: the masked coordinate keeps only low bits of the
            // 64-bit sum, which the 32-bit sum of the addends' low words already has
            const uint32_t xm = ((uint32_t)abs_x + (uint32_t)ox + (uint32_t)f->stbn_offset_x) & (uint32_t)mask_w;
            const uint32_t ym =
                ((uint32_t)abs_y + (uint32_t)oy + (uint32_t)f->stbn_offset_y + (uint32_t)pitch_offset) & (uint32_t)mask_h;
            const uint8_t v = __ldg(frame_base + ((size_t)ym * (size_t)(uint32_t)f->stbn_w + xm));
            return ((float)v + 0.5f) * (1.0f / 256.0f);
        }
        const int64_t xc = (int64_t)abs_x + (int64_t)ox + (int64_t)f->stbn_offset_x;
        const int64_t yc = (int64_t)abs_y + (int64_t)oy + (int64_t)f->stbn_offset_y + pitch_offset;
        const int x = wrap_coordinate(xc, f->stbn_w);
        const int y = wrap_coordinate(yc, f->stbn_h);
        const uint8_t v = __ldg(f->stbn + ((frame_row_base + (size_t)y) * (size_t)f->stbn_w + (size_t)x));
        return ((float)v + 0.5f) * (1.0f / 256.0f);
    }

    __device__ __forceinline__ float uniform() {
        if (use_stbn) return stbn_at(draw++);
        // u01: x * 2^-32 + 2^-33 (the product is exact, so the fma is too)
        return __fmaf_rn((float)philox.next(), 1.0f / 4294967296.0f, 0.5f / 4294967296.0f);
    }

    __device__ __forceinline__ float normal() {
        float u1 = uniform();
        u1 = clamp01(u1, 1e-7f, 1.0f);
        const float u2 = uniform();
        const float r = sqrtf(-2.0f * logf(u1));
        return r * cosf(kTwoPi * u2);
    }
};

constexpr int kStbnBatch = 4;

__device__ __forceinline__ int poisson(float lambda, GrainRng& rng) {
    if (!finite(lambda) || !(lambda > 0.0f)) return 0;
    if (lambda < 10.0f) {
        const float L = expf(-lambda);
        float p = 1.0f;
        int k = 0;
        if (rng.use_stbn) {
            // The same draws in the same order, fetched kStbnBatch at a time: the
            // blue-noise addresses do not depend on earlier draws, so the table loads
            // overlap instead of paying one cache latency per draw. Draws fetched past
            // the stop are not consumed (the draw index advances by the draws used).
            while (p > L && k < 1024) {
                float u[kStbnBatch];
#pragma unroll
                for (int j = 0; j < kStbnBatch; ++j) u[j] = rng.stbn_at(rng.draw + (uint32_t)j);
                uint32_t used = 0;
#pragma unroll
                for (int j = 0; j < kStbnBatch; ++j) {
                    if (p > L && k < 1024) {
                        ++k;
                        ++used;
                        p *= clamp01(u[j], 1e-7f, 1.0f);
                    }
                }
                rng.draw += used;
            }
            return k - 1;
        }
        while (p > L && k < 1024) {
            ++k;
            p *= clamp01(rng.uniform(), 1e-7f, 1.0f);
        }
        return k - 1;
    }
    const float z = rng.normal();
    float s = __fmaf_rn(sqrtf(lambda), z, lambda);
    if (!finite(s)) s = 0.0f;
    int k = (int)floorf(s + 0.5f);
    return k < 0 ? 0 : k;
}

struct ParticleSample {
    float density, density_max, n_particles, od_particle, uniformity;
    uint64_t seed;
    int frame_offset;
};

__device__ __forceinline__ float particle_model(const GrainFrame* f, const ParticleSample& s, uint64_t ax,
                                                uint64_t ay, int use_stbn, int wang_x, int wang_y) {
    float density = s.density;
    if (!finite(density) || density < 0.0f) density = 0.0f;
    float p = density / s.density_max;
    p = clamp01(p, 1e-6f, 1.0f - 1e-6f);
    const float u = finite(s.uniformity) ? clamp01(s.uniformity, 0.0f, 1.0f) : 0.0f;
    float sat = __fmaf_rn(-(p * u), 1.0f - 1e-6f, 1.0f);
    if (!finite(sat) || sat <= 0.0f) sat = 1e-6f;
    GrainRng rng(f, s.seed, ax, ay, use_stbn, s.frame_offset, wang_x, wang_y);
    const float lambda = s.n_particles / sat;
    const int count = poisson(lambda * p, rng);
    return sanitize((float)count * s.od_particle * sat);
}

__device__ __forceinline__ void wang_offsets(const GrainFrame* f, uint64_t ax, uint64_t ay, int& ox, int& oy) {
    ox = 0;
    oy = 0;
    if (!f->wang_tiles || !f->wang_lut || f->wang_w <= 0 || f->wang_h <= 0 || f->wang_count <= 0) return;
    if (!(f->pixel_size_um > 0.0f) || !(f->wang_cell_mm > 0.0f)) return;
    const float xmm = (float)ax * (f->pixel_size_um * 0.001f);
    const float ymm = (float)ay * (f->pixel_size_um * 0.001f);
    const float inv = 1.0f / f->wang_cell_mm;
    const float cx = xmm * inv, cy = ymm * inv;
    const float fx = cx - floorf(cx), fy = cy - floorf(cy);
    const int64_t mx = (int64_t)floorf(cx), my = (int64_t)floorf(cy);
    if (f->wang_colors <= 0) return;
    const int colors = f->wang_colors;
    const uint64_t s0 = f->clip_token != 0 ? f->clip_token : f->session_seed;
    const uint64_t base = s0 != 0 ? s0 : 1ULL;
    const uint32_t l = hash_u32((int)mx, (int)my, base, 0xA5A5A5A5u) % colors;
    const uint32_t r = hash_u32((int)(mx + 1), (int)my, base, 0x5A5A5A5Au) % colors;
    const uint32_t t = hash_u32((int)mx, (int)my, base, 0xC3C3C3C3u) % colors;
    const uint32_t b = hash_u32((int)mx, (int)(my + 1), base, 0x3C3C3C3Cu) % colors;
    const size_t c = (size_t)colors;
    const int tile = (int)f->wang_lut[(((size_t)l * c + r) * c + t) * c + b];
    const int w = f->wang_w, h = f->wang_h;
    int tx = (int)floorf(fx * (float)w), ty = (int)floorf(fy * (float)h);
    if (tx >= w) tx = w - 1;
    if (ty >= h) ty = h - 1;
    auto sample = [&](int x, int y) -> float {
        if (tile < 0 || tile >= f->wang_count) return 0.0f;
        x = x < 0 ? 0 : (x >= w ? w - 1 : x);
        y = y < 0 ? 0 : (y >= h ? h - 1 : y);
        const uint8_t v = f->wang_tiles[((size_t)tile * (size_t)h + (size_t)y) * (size_t)w + (size_t)x];
        return ((float)v + 0.5f) * (1.0f / 256.0f);
    };
    const float v0 = sample(tx, ty);
    const float v1 = sample((tx + (w >> 1)) % w, (ty + (h >> 1)) % h);
    const int warp_x = f->stbn_w > 0 ? ((f->stbn_w / 8) > 4 ? f->stbn_w / 8 : 4) : 0;
    const int warp_y = f->stbn_h > 0 ? ((f->stbn_h / 8) > 4 ? f->stbn_h / 8 : 4) : 0;
    if (warp_x == 0 || warp_y == 0) return;
    ox = (int)floorf((v0 - 0.5f) * 2.0f * (float)warp_x);
    oy = (int)floorf((v1 - 0.5f) * 2.0f * (float)warp_y);
}

__device__ __forceinline__ float breathing_factor(const GrainFrame* f, const GrainFrameUniforms& u, uint64_t ax,
                                                  uint64_t ay) {
    if (!u.breathing_active) return 1.0f;
    const float bx = (float)ax + u.breathing_drift_x;
    const float by = (float)ay + u.breathing_drift_y + u.breathing_roll_y;
    const float xs = bx / u.breathing_cell_small_px, ys = by / u.breathing_cell_small_px;
    const float xl = bx / u.breathing_cell_large_px, yl = by / u.breathing_cell_large_px;
    const float sa = value_noise(xs, ys, u.breathing_seed_a ^ 0x9E3779B97F4A7C15ULL);
    const float sb = value_noise(xs, ys, u.breathing_seed_b ^ 0x9E3779B97F4A7C15ULL);
    const float la = value_noise(xl, yl, u.breathing_seed_a ^ 0xBF58476D1CE4E5B9ULL);
    const float lb = value_noise(xl, yl, u.breathing_seed_b ^ 0xBF58476D1CE4E5B9ULL);
    const float ns = __fmaf_rn(sb - sa, u.breathing_t, sa);
    const float nl = __fmaf_rn(lb - la, u.breathing_t, la);
    const float noise = __fmaf_rn(u.breathing_mix, ns, (1.0f - u.breathing_mix) * nl);
    const float n = __fmaf_rn(noise, 2.0f, -1.0f);
    const float factor = __fmaf_rn(f->breathing_amplitude, n, 1.0f);
    return factor > 0.0f ? factor : 0.0f;
}

__device__ __forceinline__ float clump_factor(const GrainFrameUniforms& u, uint64_t ax, uint64_t ay) {
    if (!u.clump_active) return 1.0f;
    const float bx = (float)ax;
    const float by = (float)ay + u.clump_roll_y;
    const float xs = bx / u.clump_cell_px, ys = by / u.clump_cell_px;
    const float a = value_noise(xs, ys, u.clump_static_seed ^ 0x9E3779B97F4A7C15ULL);
    const float b = value_noise(xs + 19.19f, ys + 7.23f, u.clump_static_seed ^ 0xBF58476D1CE4E5B9ULL);
    const float u1 = clamp01(a, 1e-6f, 1.0f - 1e-6f);
    const float u2 = clamp01(b, 0.0f, 1.0f);
    const float r = sqrtf(-2.0f * logf(u1));
    const float n = r * cosf(kTwoPi * u2);
    float v = expf(__fmaf_rn(u.clump_sigma, n, u.clump_mu));
    if (!finite(v)) v = 1.0f;
    return v * u.clump_rms_norm;
}

// Density of one sublayer at the given total density: linear interpolation of the
// layer curve over the capture density curve (negated for positive film), with the
// 16-block prefix-maximum search for finite 256-sample axes.
__device__ float layer_density(const GrainFrame* f, int ch, int layer, float density) {
    const float* x = f->base_curve[ch];
    const float* y = f->layer_curve[layer][ch];
    const int n = f->base_curve_n[ch];
    if (!x || !y || n <= 0) return density;
    if (!finite(density)) return __ldg(y);
    const bool pos = f->positive_film != 0;
    const float q = pos ? -density : density;
    auto axis = [&](int i) {
        const float v = __ldg(x + i);
        return pos ? -v : v;
    };
    const bool bounded = f->axis_finite[ch] != 0 && n == 256;
    int b0 = 0, b1 = n - 1;
    if (!bounded) {
        while (b0 < n && !finite(axis(b0))) ++b0;
        if (b0 >= n) return density;
        while (b1 > b0 && !finite(axis(b1))) --b1;
    }
    const float xmin = axis(b0), xmax = axis(b1);
    if (!finite(xmin) || !finite(xmax) || !(xmax >= xmin)) return __ldg(y + b0);
    if (q <= xmin) return __ldg(y + b0);
    if (q >= xmax) return __ldg(y + b1);
    int i1 = b0 + 1;
    if (bounded) {
        const float* prefix = f->axis_block_prefix_max[ch];
        int lo = 0, hi = 15;
#pragma unroll
        for (int step = 0; step < 4; ++step) {
            const int mid = lo + (hi - lo) / 2;
            if (prefix[mid] < q)
                lo = mid + 1;
            else
                hi = mid;
        }
        i1 = max(1, lo * 16);
        const int end = min(b1, (lo + 1) * 16 - 1);
        while (i1 <= end && axis(i1) < q) ++i1;
    } else {
        while (i1 <= b1 && axis(i1) < q) ++i1;
    }
    if (i1 > b1) return __ldg(y + b1);
    const int i0 = i1 - 1;
    const float x0 = axis(i0), x1v = axis(i1);
    const float y0 = __ldg(y + i0), y1 = __ldg(y + i1);
    const float den = x1v - x0;
    if (!(den > 0.0f) || !finite(den)) return y0;
    const float t = (q - x0) / den;
    return __fmaf_rn(t, y1 - y0, y0);
}

struct PixelContext {
    uint64_t ax, ay;
    int use_stbn, wang_x, wang_y;
    float breathing, clump;
    bool retime;
    float time_alpha;
};

// One layer's particle sample with the breathing/clump modulation and retiming.
__device__ __forceinline__ float modulated_sample(const GrainFrame* f, const PixelContext& px, ParticleSample s,
                                                  uint64_t seed_next) {
    const float density = s.density;
    float g = particle_model(f, s, px.ax, px.ay, px.use_stbn, px.wang_x, px.wang_y);
    float gn = 0.0f;
    if (px.retime) {
        s.seed = seed_next;
        s.frame_offset = 1;
        gn = particle_model(f, s, px.ax, px.ay, px.use_stbn, px.wang_x, px.wang_y);
    }
    g = __fmaf_rn((g - density) * px.breathing, px.clump, density);
    if (px.retime) {
        gn = __fmaf_rn((gn - density) * px.breathing, px.clump, density);
        const float d0 = g - density, d1 = gn - density;
        const float blend = __fmaf_rn(d1 - d0, px.time_alpha, d0);
        const float w0 = 1.0f - px.time_alpha;
        const float den = __fmaf_rn(w0, w0, px.time_alpha * px.time_alpha) + 1e-6f;
        g = __fmaf_rn(blend, rsqrtf(den), density);
    }
    return g;
}

template <int Mode>
__global__ void __launch_bounds__(256) grain_sample_kernel(const __grid_constant__ GrainFrame f, int ch, int layer,
                                                           const float* __restrict__ density_in, long long din_stride,
                                                           GrainPlane out, GrainSampleEpilogue ep, int width,
                                                           int height) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    const GrainFrameUniforms u = *f.uniforms;
    const float in_density = density_in[(long long)y * din_stride + x];
    PixelContext px;
    px.ax = (uint64_t)((int64_t)f.origin_x + x);
    px.ay = (uint64_t)((int64_t)f.origin_y + y);
    px.time_alpha = f.time_alpha;
    px.retime = f.time_alpha > 1e-6f && f.time_alpha < 0.999999f;
    px.use_stbn = (f.stbn && f.stbn_w > 0 && f.stbn_h > 0 && f.stbn_frames > 0) ? 1 : 0;
    px.wang_x = px.wang_y = 0;
    px.clump = clump_factor(u, px.ax, px.ay);
    if (px.use_stbn) wang_offsets(&f, px.ax, px.ay, px.wang_x, px.wang_y);
    px.breathing = breathing_factor(&f, u, px.ax, px.ay);

    float value;
    if (Mode == kGrainSimple) {
        const float density = in_density + f.density_min[ch];
        const int nsub = f.n_sublayers > 0 ? f.n_sublayers : 1;
        float acc = 0.0f, accn = 0.0f;
        for (int sl = 0; sl < nsub; ++sl) {
            const uint64_t salt = (uint64_t)ch + (uint64_t)sl * 10ULL;
            ParticleSample s{density, f.density_max[ch], f.n_particles[ch], f.od_particle[ch], f.uniformity[ch],
                             f.seed_base ^ salt, 0};
            acc += particle_model(&f, s, px.ax, px.ay, px.use_stbn, px.wang_x, px.wang_y);
            if (px.retime) {
                s.seed = f.seed_base_next ^ salt;
                s.frame_offset = 1;
                accn += particle_model(&f, s, px.ax, px.ay, px.use_stbn, px.wang_x, px.wang_y);
            }
        }
        acc /= (float)nsub;
        if (px.retime) accn /= (float)nsub;
        acc = __fmaf_rn((acc - density) * px.breathing, px.clump, density);
        if (px.retime) {
            accn = __fmaf_rn((accn - density) * px.breathing, px.clump, density);
            const float d0 = acc - density, d1 = accn - density;
            const float blend = __fmaf_rn(d1 - d0, px.time_alpha, d0);
            const float w0 = 1.0f - px.time_alpha;
            const float den = __fmaf_rn(w0, w0, px.time_alpha * px.time_alpha) + 1e-6f;
            acc = __fmaf_rn(blend, rsqrtf(den), density);
        }
        value = sanitize(acc);
    } else if (Mode == kGrainLayer) {
        const float density = layer_density(&f, ch, layer, in_density) + f.density_min_layers[layer][ch];
        const uint64_t salt = (uint64_t)ch + (uint64_t)layer * 10ULL;
        const ParticleSample s{density,
                               f.density_max_layers[layer][ch],
                               f.n_particles_layers[layer][ch],
                               f.od_particle_layers[layer][ch],
                               f.uniformity[ch],
                               f.seed_base ^ salt,
                               0};
        value = sanitize(modulated_sample(&f, px, s, f.seed_base_next ^ salt));
    } else {
        float sum = 0.0f;
        for (int l = 0; l < 3; ++l) {
            const float density = layer_density(&f, ch, l, in_density) + f.density_min_layers[l][ch];
            const uint64_t salt = (uint64_t)ch + (uint64_t)l * 10ULL;
            const ParticleSample s{density,
                                   f.density_max_layers[l][ch],
                                   f.n_particles_layers[l][ch],
                                   f.od_particle_layers[l][ch],
                                   f.uniformity[ch],
                                   f.seed_base ^ salt,
                                   0};
            sum += sanitize(modulated_sample(&f, px, s, f.seed_base_next ^ salt));
        }
        value = sanitize(sum);
    }

    float* o = out.p + (long long)y * out.stride + x;
    if (ep.accumulate) value = sanitize((ep.init ? 0.0f : *o) + value);
    if (ep.form_delta) {
        if (ep.density_bias != 0.0f) value = sanitize(value + ep.density_bias);
        value = sanitize(value - in_density);
    }
    *o = value;
}

__device__ __forceinline__ int reflect_half(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * n;
    int m = i % period;
    if (m < 0) m += period;
    return m < n ? m : period - 1 - m;
}

constexpr int kRowTile = 128;
constexpr int kRowLines = 4;

__global__ void __launch_bounds__(kRowTile* kRowLines) grain_rows_kernel(const float* __restrict__ in,
                                                                        long long in_stride, float* __restrict__ out,
                                                                        long long out_stride,
                                                                        const __grid_constant__ GrainBlurTaps taps,
                                                                        int width, int height) {
    extern __shared__ float tile[];
    const int r = taps.radius;
    const int tw = kRowTile + 2 * r;
    const int x0 = blockIdx.x * kRowTile;
    const int y = blockIdx.y * kRowLines + threadIdx.y;
    float* row = tile + threadIdx.y * tw;
    if (y < height) {
        const float* src = in + (long long)y * in_stride;
        for (int i = threadIdx.x; i < tw; i += kRowTile) row[i] = src[reflect_half(x0 - r + i, width)];
    }
    __syncthreads();
    const int x = x0 + threadIdx.x;
    if (y >= height || x >= width) return;
    float acc = 0.0f;
    const float* v = row + threadIdx.x;
    for (int k = 0; k <= 2 * r; ++k) acc = __fmaf_rn(v[k], taps.w[k], acc);
    out[(long long)y * out_stride + x] = sanitize(acc);
}

constexpr int kColTileX = 32;
constexpr int kColTileY = 32;
constexpr int kColThreadsY = 8;

__global__ void __launch_bounds__(kColTileX* kColThreadsY) grain_columns_kernel(
    const float* __restrict__ in, long long in_stride, GrainPlane out, const __grid_constant__ GrainBlurTaps taps,
    GrainVerticalEpilogue ep, int width, int height) {
    extern __shared__ float tile[];
    const int r = taps.radius;
    const int th = kColTileY + 2 * r;
    const int x0 = blockIdx.x * kColTileX, y0 = blockIdx.y * kColTileY;
    const int x = x0 + threadIdx.x;
    if (x < width)
        for (int i = threadIdx.y; i < th; i += kColThreadsY)
            tile[i * kColTileX + threadIdx.x] = in[(long long)reflect_half(y0 - r + i, height) * in_stride + x];
    __syncthreads();
    if (x >= width) return;
    const float w = isfinite(ep.weight) ? ep.weight : 0.0f;
    const float gain = isfinite(ep.gain) ? ep.gain : 0.0f;
    for (int j = threadIdx.y; j < kColTileY; j += kColThreadsY) {
        const int y = y0 + j;
        if (y >= height) break;
        float acc = 0.0f;
        const float* v = tile + j * kColTileX + threadIdx.x;
        for (int k = 0; k <= 2 * r; ++k) acc = __fmaf_rn(v[k * kColTileX], taps.w[k], acc);
        const float blurred = sanitize(acc);
        float* o = out.p + (long long)y * out.stride + x;
        const float prev = ep.init ? 0.0f : *o;
        float value = ep.weighted ? __fmaf_rn(w, blurred, prev) : prev + blurred;
        value = sanitize(value);
        if (!ep.weighted && ep.density) {
            if (ep.density_bias != 0.0f) value = sanitize(value + ep.density_bias);
            value = sanitize(value - ep.density[(long long)y * ep.density_stride + x]);
        }
        if (ep.apply_gain) value = sanitize(value * gain);
        *o = value;
    }
}

__global__ void grain_accumulate_weighted_kernel(GrainPlane dst, const float* __restrict__ src, long long src_stride,
                                                 float weight, int init, int apply_gain, float gain, int width,
                                                 int height) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    const float w = isfinite(weight) ? weight : 0.0f;
    float* o = dst.p + (long long)y * dst.stride + x;
    float v = sanitize(__fmaf_rn(w, src[(long long)y * src_stride + x], init ? 0.0f : *o));
    if (apply_gain) v = sanitize(v * (isfinite(gain) ? gain : 0.0f));
    *o = v;
}

__global__ void grain_clear_kernel(GrainPlane dst, int width, int height) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < width && y < height) dst.p[(long long)y * dst.stride + x] = 0.0f;
}

__global__ void grain_finish_kernel(float* density, long long density_stride, const float* __restrict__ delta,
                                    long long delta_stride, const float* __restrict__ shared, float shared_weight,
                                    float independent_weight, float amplitude, float scale, int add_mean, int width,
                                    int height) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || y >= height) return;
    const long long di = (long long)y * delta_stride + x;
    float d;
    if (shared) {
        // the independent delta is read only when it carries weight (it is not
        // generated otherwise)
        const float sw = clamp01(shared_weight, 0.0f, 1.0f);
        const float iw = clamp01(independent_weight, 0.0f, 1.0f);
        const float sv = sw > 0.0f ? shared[di] : 0.0f;
        const float iv = iw > 0.0f ? delta[di] : 0.0f;
        d = sanitize(amplitude * __fmaf_rn(sw, sv, iw * iv));
    } else {
        d = delta[di];
    }
    float* o = density + (long long)y * density_stride + x;
    const float s = isfinite(scale) ? scale : 0.0f;
    const float mean = add_mean ? *o : 0.0f;
    *o = sanitize(__fmaf_rn(s, d, mean));
}

__global__ void grain_debug_average_kernel(float* c, float* m, float* y, long long stride, float offset, float scale,
                                           int width, int height) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int yy = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= width || yy >= height) return;
    const long long i = (long long)yy * stride + x;
    const float s = isfinite(scale) ? scale : 1.0f;
    const float o = isfinite(offset) ? offset : 0.0f;
    float avg = (c[i] + m[i] + y[i]) * (1.0f / 3.0f);
    if (!isfinite(avg)) avg = 0.0f;
    const float v = __fmaf_rn(avg, s, o);
    c[i] = v;
    m[i] = v;
    y[i] = v;
}

struct LognormalParameters {
    float mu, sigma;
};

__device__ __forceinline__ LognormalParameters lognormal_from_mean_std(float mean, float sd) {
    const float m2 = mean * mean, s2 = sd * sd;
    const float sigma_sq = logf(1.0f + s2 / m2);
    return {__fmaf_rn(-0.5f, sigma_sq, logf(fmaxf(1e-12f, mean))), sqrtf(fmaxf(0.0f, sigma_sq))};
}

__global__ void grain_uniforms_kernel(const __grid_constant__ GrainFrame f) {
    if (blockIdx.x != 0 || threadIdx.x != 0 || !f.uniforms) return;
    GrainFrameUniforms u{};
    const float time = (float)f.frame_index + f.time_alpha;
    if (f.breathing_amplitude > 0.0f && f.breathing_period_frames > 0 && f.pixel_size_um > 0.0f &&
        f.breathing_cell_um_small > 0.0f && f.breathing_cell_um_large > 0.0f) {
        const float period = (float)f.breathing_period_frames;
        const float step_f = floorf(time / period);
        const int64_t step = (int64_t)step_f;
        const float frac = __fmaf_rn(-step_f, period, time) / period;
        u.breathing_t = smoothstep(clamp01(frac, 0.0f, 1.0f));
        const uint64_t seed = f.session_seed != 0 ? f.session_seed : 1ULL;
        u.breathing_seed_a = splitmix64(seed ^ ((uint64_t)step * 0x8EBC6AF09C88C6E3ULL));
        u.breathing_seed_b = splitmix64(seed ^ ((uint64_t)(step + 1) * 0x8EBC6AF09C88C6E3ULL));
        const float inv_px = 1.0f / f.pixel_size_um;
        u.breathing_cell_small_px = fmaxf(4.0f, f.breathing_cell_um_small * inv_px);
        u.breathing_cell_large_px = fmaxf(4.0f, f.breathing_cell_um_large * inv_px);
        float drift = 0.0f;
        if (f.breathing_drift_um_per_frame > 0.0f) drift = f.breathing_drift_um_per_frame * inv_px;
        float dx = 0.0f, dy = 0.0f;
        if (drift > 0.0f) {
            const uint64_t h = splitmix64(seed ^ 0x6A09E667F3BCC909ULL);
            const float angle = (float)(uint32_t)(h & 0xFFFFFFFFu) * kInvU32 * kTwoPi;
            dx = cosf(angle) * drift;
            dy = sinf(angle) * drift;
        }
        const float roll = f.pitch_px > 0 ? (float)f.pitch_px : 0.0f;
        u.breathing_drift_x = dx * time;
        u.breathing_drift_y = dy * time;
        u.breathing_roll_y = roll * time;
        u.breathing_mix = clamp01(f.breathing_mix, 0.0f, 1.0f);
        u.breathing_active = 1;
    }
    const float sd_spatial = f.micro_structure[1] * 0.001f;
    if (sd_spatial > 0.0f && f.pixel_size_um > 0.0f) {
        float cell_um = f.micro_structure[0];
        if (!(cell_um > 0.0f)) cell_um = 0.0f;
        const float inv_px = 1.0f / f.pixel_size_um;
        u.clump_cell_px = cell_um * inv_px;
        if (!(u.clump_cell_px > 4.0f)) u.clump_cell_px = 4.0f;
        const float roll = f.pitch_px > 0 ? (float)f.pitch_px : 0.0f;
        u.clump_roll_y = roll * time;
        u.clump_static_seed = f.clip_token != 0 ? f.clip_token : f.session_seed;
        if (u.clump_static_seed == 0) u.clump_static_seed = 1ULL;
        float sd = sd_spatial;
        u.clump_rms_norm = 1.0f;
        const float mix = clamp01(f.clump_temporal_mix, 0.0f, 1.0f);
        if (mix > 0.0f) {
            int period_i = f.clump_morph_period_frames;
            if (period_i <= 0) period_i = 1;
            const float period = (float)period_i;
            const float step_f = floorf(time / period);
            const int64_t step = (int64_t)step_f;
            const float frac = __fmaf_rn(-step_f, period, time) / period;
            const float t = smoothstep(clamp01(frac, 0.0f, 1.0f));
            const uint64_t tseed = f.session_seed != 0 ? f.session_seed : 1ULL;
            const uint64_t sa = splitmix64(tseed ^ ((uint64_t)step * 0xD2B74407B1CE6E93ULL));
            const uint64_t sb = splitmix64(tseed ^ ((uint64_t)(step + 1) * 0xD2B74407B1CE6E93ULL));
            const float u1a = hash01(0, 0, sa ^ 0x9E3779B97F4A7C15ULL);
            const float u2a = hash01(1, 0, sa ^ 0xBF58476D1CE4E5B9ULL);
            const float u1b = hash01(0, 0, sb ^ 0x9E3779B97F4A7C15ULL);
            const float u2b = hash01(1, 0, sb ^ 0xBF58476D1CE4E5B9ULL);
            float u1 = __fmaf_rn(u1b - u1a, t, u1a);
            float u2 = __fmaf_rn(u2b - u2a, t, u2a);
            u1 = clamp01(u1, 1e-6f, 1.0f - 1e-6f);
            u2 = clamp01(u2, 0.0f, 1.0f);
            const float rt = sqrtf(-2.0f * logf(u1));
            const float nt = rt * cosf(kTwoPi * u2);
            const float strength_sd = mix * 0.23597824f;
            const LognormalParameters lp = lognormal_from_mean_std(1.0f, strength_sd);
            float strength = expf(__fmaf_rn(lp.sigma, nt, lp.mu));
            strength *= rsqrtf(__fmaf_rn(strength_sd, strength_sd, 1.0f));
            sd = sd_spatial * strength;
            const float den = __fmaf_rn(sd, sd, 1.0f);
            const float num = __fmaf_rn(sd_spatial, sd_spatial, 1.0f);
            u.clump_rms_norm = den > 0.0f ? sqrtf(num / den) : 1.0f;
        }
        const LognormalParameters lp = lognormal_from_mean_std(1.0f, sd);
        u.clump_mu = lp.mu;
        u.clump_sigma = lp.sigma;
        u.clump_active = 1;
    }
    *f.uniforms = u;
}

dim3 plane_grid(int width, int height) { return dim3((width + 31) / 32, (height + 7) / 8); }

} // namespace

cudaError_t launch_grain_uniforms(const GrainFrame& f, cudaStream_t s) {
    fjb::count_launch();
    grain_uniforms_kernel<<<1, 32, 0, s>>>(f);
    return cudaGetLastError();
}

cudaError_t launch_grain_sample(const GrainFrame& f, int mode, int channel, int layer, const float* density,
                                long long density_stride, GrainPlane out, const GrainSampleEpilogue& ep, int width,
                                int height, cudaStream_t s) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    const dim3 block(32, 8), grid = plane_grid(width, height);
    switch (mode) {
    case kGrainSimple:
        fjb::count_launch();
        grain_sample_kernel<kGrainSimple><<<grid, block, 0, s>>>(f, channel, layer, density, density_stride, out, ep,
                                                                 width, height);
        break;
    case kGrainLayer:
        fjb::count_launch();
        grain_sample_kernel<kGrainLayer><<<grid, block, 0, s>>>(f, channel, layer, density, density_stride, out, ep,
                                                                width, height);
        break;
    default:
        fjb::count_launch();
        grain_sample_kernel<kGrainTriplet><<<grid, block, 0, s>>>(f, channel, layer, density, density_stride, out,
                                                                  ep, width, height);
        break;
    }
    return cudaGetLastError();
}

cudaError_t launch_grain_blur_rows(const float* in, long long in_stride, float* out, long long out_stride,
                                   const GrainBlurTaps& taps, int width, int height, cudaStream_t s) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    if (taps.radius <= 0 || taps.radius > kGrainMaxRadius) return cudaErrorInvalidValue;
    const size_t smem = (size_t)kRowLines * (kRowTile + 2 * taps.radius) * sizeof(float);
    const dim3 grid((width + kRowTile - 1) / kRowTile, (height + kRowLines - 1) / kRowLines);
    fjb::count_launch();
    grain_rows_kernel<<<grid, dim3(kRowTile, kRowLines), smem, s>>>(in, in_stride, out, out_stride, taps, width,
                                                                    height);
    return cudaGetLastError();
}

cudaError_t launch_grain_blur_columns(const float* in, long long in_stride, GrainPlane out,
                                      const GrainBlurTaps& taps, const GrainVerticalEpilogue& ep, int width,
                                      int height, cudaStream_t s) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    if (taps.radius <= 0 || taps.radius > kGrainMaxRadius) return cudaErrorInvalidValue;
    const size_t smem = (size_t)(kColTileY + 2 * taps.radius) * kColTileX * sizeof(float);
    const dim3 grid((width + kColTileX - 1) / kColTileX, (height + kColTileY - 1) / kColTileY);
    fjb::count_launch();
    grain_columns_kernel<<<grid, dim3(kColTileX, kColThreadsY), smem, s>>>(in, in_stride, out, taps, ep, width,
                                                                           height);
    return cudaGetLastError();
}

cudaError_t launch_grain_accumulate_weighted(GrainPlane dst, const float* src, long long src_stride, float weight,
                                             int init, int apply_gain, float gain, int width, int height,
                                             cudaStream_t s) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    fjb::count_launch();
    grain_accumulate_weighted_kernel<<<plane_grid(width, height), dim3(32, 8), 0, s>>>(
        dst, src, src_stride, weight, init, apply_gain, gain, width, height);
    return cudaGetLastError();
}

cudaError_t launch_grain_clear(GrainPlane dst, int width, int height, cudaStream_t s) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    fjb::count_launch();
    grain_clear_kernel<<<plane_grid(width, height), dim3(32, 8), 0, s>>>(dst, width, height);
    return cudaGetLastError();
}

cudaError_t launch_grain_finish(float* density, long long density_stride, const float* delta, long long delta_stride,
                                const float* shared, float shared_weight, float independent_weight, float amplitude,
                                float scale, int add_mean, int width, int height, cudaStream_t s) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    fjb::count_launch();
    grain_finish_kernel<<<plane_grid(width, height), dim3(32, 8), 0, s>>>(
        density, density_stride, delta, delta_stride, shared, shared_weight, independent_weight, amplitude, scale,
        add_mean, width, height);
    return cudaGetLastError();
}

cudaError_t launch_grain_debug_average(float* c, float* m, float* y, long long stride, float offset, float scale,
                                       int width, int height, cudaStream_t s) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    fjb::count_launch();
    grain_debug_average_kernel<<<plane_grid(width, height), dim3(32, 8), 0, s>>>(c, m, y, stride, offset, scale,
                                                                                width, height);
    return cudaGetLastError();
}

} // namespace fjb
