// fjb_tc_lut.cu -- the film TC LUT built on the device (per-recipe precompute).
//
// Restates rust/film-juicer-core/src/reconstruction.rs: build_tc_lut (:594-677) for the
// Hanatos irradiance method, with its optional spectral blur (blur_spectra :540-569,
// gaussian_kernel :227-268, gaussian_reflect_index :270-279), and the Arctic reflectance
// method with its neutral-response denominators (sample_mitchell :501-538 at the
// projected white, projected_white :124-137). The host code rounds every float product
// and sum on its own (Rust does not fuse), so the kernels spell each one out with
// __fmul_rn / __fadd_rn / __fdiv_rn: the table is the reference's word for word.
// The Hanatos surface correction (eval_hanatos_surface :570-593) is a factor per node
// and channel: exp2 of a polynomial in the node's offset from the projected white,
// evaluated on the host with the C library's exp2f (what f32::exp2 calls) and applied
// on the device. The input-compression remap (gamut.rs:259-373) moves every node to the
// coordinates of its compressed chromaticity: those depend only on the input hull, so
// the host computes them in FP64 with the C library's hypot and pow (as the Rust host
// does) and the device resamples the table bilinearly, unfused, at them.
//
// B200 schedule: one thread per (c, m) node, the 81 wavelengths (blurred on the fly
// when the blur is on, each tap in the reference's order) contracted with the
// sensitivity into three sums; the tables it reads (sensitivity, illuminant, blur taps)
// are kernel parameters, i.e. in the constant bank. 36 864 nodes x 81 x 3 products.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "fjb_launches.h"
#include "fjb_schedule.h"

namespace fjb {

namespace {

constexpr int kNodes = 192 * 192;
constexpr int kMaxBlurTaps = 161; // radius 80: wider kernels fold onto the 81 samples anyway
constexpr unsigned kBlurNonFinite = 1u, kIntegratedNonFinite = 2u, kNeutralInvalid = 4u, kSamplingUnusable = 8u,
                   kRemappedNonFinite = 16u;

struct TcParams {
    float sens[81 * 3];
    float illum[81];
    float taps[kMaxBlurTaps];
    int radius; // 0: no blur
    int arctic;
    float tc_c, tc_m; // projected white (Arctic)
};

__device__ __forceinline__ int reflect81(int i) {
    int r = i % 162;
    if (r < 0) r += 162;
    return r >= 81 ? 161 - r : r;
}

__device__ __forceinline__ float spectral_sample(const float* __restrict__ node, const TcParams& p, int s) {
    if (p.radius == 0) return __ldg(node + s);
    float v = 0.0f;
    for (int k = 0; k <= 2 * p.radius; ++k) v = __fadd_rn(v, __fmul_rn(p.taps[k], __ldg(node + reflect81(s + k - p.radius))));
    return v;
}

// Mitchell-Netravali (B = C = 1/3) weight with every product and sum rounded alone.
__device__ float mitchell_unfused(float t) {
    const float B = 1.0f / 3.0f, C = 1.0f / 3.0f;
    const float x = fabsf(t);
    if (x < 1.0f) {
        const float a = __fadd_rn(__fadd_rn(12.0f, -__fmul_rn(9.0f, B)), -__fmul_rn(6.0f, C));
        const float b = __fadd_rn(__fadd_rn(-18.0f, __fmul_rn(12.0f, B)), __fmul_rn(6.0f, C));
        const float c = __fadd_rn(6.0f, -__fmul_rn(2.0f, B));
        const float s = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(__fmul_rn(a, x), x), x), __fmul_rn(__fmul_rn(b, x), x)), c);
        return __fmul_rn(1.0f / 6.0f, s);
    }
    if (x < 2.0f) {
        const float a = __fadd_rn(-B, -__fmul_rn(6.0f, C));
        const float b = __fadd_rn(__fmul_rn(6.0f, B), __fmul_rn(30.0f, C));
        const float c = __fadd_rn(__fmul_rn(-12.0f, B), -__fmul_rn(48.0f, C));
        const float d = __fadd_rn(__fmul_rn(8.0f, B), __fmul_rn(24.0f, C));
        const float s = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(__fmul_rn(a, x), x), x),
                                                      __fmul_rn(__fmul_rn(b, x), x)),
                                            __fmul_rn(c, x)),
                                  d);
        return __fmul_rn(1.0f / 6.0f, s);
    }
    return 0.0f;
}

__device__ void mitchell_coord(float v, int& base, float& frac) {
    v = __fmul_rn(fminf(fmaxf(v, 0.0f), 1.0f), 191.0f);
    if (v >= 191.0f) {
        base = 190;
        frac = 1.0f;
        return;
    }
    base = (int)floorf(v);
    frac = __fadd_rn(v, -(float)base);
}

__device__ __forceinline__ int reflect192(int i) { return i < 0 ? -i : (i >= 192 ? 382 - i : i); }

// Neutral response of the Arctic method: the projected white's reflectance spectrum
// (Mitchell-interpolated) relit by the illuminant and integrated per channel.
__global__ void tc_neutral_kernel(const float* __restrict__ spectra, const __grid_constant__ TcParams p, float* den,
                                  unsigned* flags) {
    int cb, mb;
    float cf, mf;
    mitchell_coord(p.tc_c, cb, cf);
    mitchell_coord(p.tc_m, mb, mf);
    const float cw[4] = {mitchell_unfused(__fadd_rn(cf, 1.0f)), mitchell_unfused(cf), mitchell_unfused(__fadd_rn(cf, -1.0f)),
                         mitchell_unfused(__fadd_rn(cf, -2.0f))};
    const float mw[4] = {mitchell_unfused(__fadd_rn(mf, 1.0f)), mitchell_unfused(mf), mitchell_unfused(__fadd_rn(mf, -1.0f)),
                         mitchell_unfused(__fadd_rn(mf, -2.0f))};
    float d[3] = {0.0f, 0.0f, 0.0f};
    for (int s = 0; s < 81; ++s) {
        float value = 0.0f, wsum = 0.0f;
        for (int dc = 0; dc < 4; ++dc) {
            const int c = reflect192(cb - 1 + dc);
            for (int dm = 0; dm < 4; ++dm) {
                const int m = reflect192(mb - 1 + dm);
                const float w = __fmul_rn(cw[dc], mw[dm]);
                wsum = __fadd_rn(wsum, w);
                value = __fadd_rn(value, __fmul_rn(w, spectra[(size_t)(c * 192 + m) * 81 + s]));
            }
        }
        const float reflectance = wsum != 0.0f ? __fdiv_rn(value, wsum) : 0.0f;
        const float relit = __fmul_rn(reflectance, p.illum[s]);
        for (int c = 0; c < 3; ++c) d[c] = __fadd_rn(d[c], __fmul_rn(relit, p.sens[s * 3 + c]));
    }
    for (int c = 0; c < 3; ++c) {
        den[c] = d[c];
        if (!(isfinite(d[c]) && d[c] > 0.0f)) atomicOr(flags, kNeutralInvalid);
    }
}

__global__ void __launch_bounds__(128) tc_lut_kernel(const float* __restrict__ spectra, const __grid_constant__ TcParams p,
                                                     const float* __restrict__ den, const float* __restrict__ surface,
                                                     float* __restrict__ table, unsigned* flags) {
    const int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= kNodes) return;
    if (p.arctic && (__ldg(flags) & kNeutralInvalid)) return;
    const float* src = spectra + (size_t)node * 81;
    float raw[3] = {0.0f, 0.0f, 0.0f};
    bool blur_bad = false;
    for (int s = 0; s < 81; ++s) {
        float e = spectral_sample(src, p, s);
        blur_bad |= p.radius > 0 && !isfinite(e);
        if (p.arctic) e = __fmul_rn(e, p.illum[s]);
        for (int c = 0; c < 3; ++c) raw[c] = __fadd_rn(raw[c], __fmul_rn(e, p.sens[s * 3 + c]));
    }
    bool bad = false;
    float4 out;
    float* o = &out.x;
    for (int c = 0; c < 3; ++c) {
        o[c] = p.arctic ? __fdiv_rn(raw[c], den[c]) : __fdiv_rn(raw[c], 1.0f);
        if (surface) o[c] = __fmul_rn(o[c], __ldg(surface + (size_t)node * 3 + c));
        bad |= !isfinite(o[c]);
    }
    out.w = 0.0f;
    reinterpret_cast<float4*>(table)[node] = out;
    if (blur_bad) atomicOr(flags, kBlurNonFinite);
    if (bad) atomicOr(flags, kIntegratedNonFinite);
}

// Bilinear resampling of the built table at each node's compressed coordinates
// (gamut.rs:324-341, every product and sum rounded alone).
__global__ void __launch_bounds__(128) tc_remap_kernel(const float* __restrict__ built, const float2* __restrict__ tc,
                                                       float* __restrict__ table, unsigned* flags) {
    const int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= kNodes) return;
    const float2 t = tc[node];
    const float cp = __fmul_rn(fminf(fmaxf(t.x, 0.0f), 1.0f), 191.0f);
    const float mp = __fmul_rn(fminf(fmaxf(t.y, 0.0f), 1.0f), 191.0f);
    if (!isfinite(cp) || !isfinite(mp)) {
        atomicOr(flags, kSamplingUnusable);
        return;
    }
    const int c0 = (int)floorf(cp), m0 = (int)floorf(mp);
    const int c1 = min(c0 + 1, 191), m1 = min(m0 + 1, 191);
    const float cf = __fadd_rn(cp, -(float)c0), mf = __fadd_rn(mp, -(float)m0);
    float4 out;
    float* o = &out.x;
    bool bad = false;
    for (int ch = 0; ch < 3; ++ch) {
        const float v00 = built[(c0 * 192 + m0) * 4 + ch], v10 = built[(c1 * 192 + m0) * 4 + ch];
        const float v01 = built[(c0 * 192 + m1) * 4 + ch], v11 = built[(c1 * 192 + m1) * 4 + ch];
        const float r0 = __fadd_rn(v00, __fmul_rn(cf, __fadd_rn(v10, -v00)));
        const float r1 = __fadd_rn(v01, __fmul_rn(cf, __fadd_rn(v11, -v01)));
        o[ch] = __fadd_rn(r0, __fmul_rn(mf, __fadd_rn(r1, -r0)));
        bad |= !isfinite(o[ch]);
    }
    out.w = 0.0f;
    reinterpret_cast<float4*>(table)[node] = out;
    if (bad) atomicOr(flags, kRemappedNonFinite);
}

// f32 arithmetic the compiler may not fuse (host side of the reference's kernel set-up)
float mul(float a, float b) {
    volatile float r = a * b;
    return r;
}
float add(float a, float b) {
    volatile float r = a + b;
    return r;
}

// exp2 of the surface polynomial per node and channel (reconstruction.rs:570-593,
// :626-660): tc = (c / 191, m / 191) about the projected white.
std::vector<float> surface_factors(const float* params, float center_c, float center_m) {
    std::vector<float> f((size_t)kNodes * 3);
    for (int c = 0; c < 192; ++c) {
        const float tcc = (float)c / 191.0f;
        for (int m = 0; m < 192; ++m) {
            const float tcm = (float)m / 191.0f;
            const float x = add(tcc, -center_c), y = add(tcm, -center_m);
            const float x2 = mul(x, x), y2 = mul(y, y), x3 = mul(x2, x), y3 = mul(y2, y);
            for (int ch = 0; ch < 3; ++ch) {
                const float* q = params + ch * 15;
                float raw = mul(q[1], x);
                raw = add(raw, mul(q[2], y));
                raw = add(raw, mul(q[3], x2));
                raw = add(raw, mul(q[4], y2));
                raw = add(raw, mul(mul(q[5], x), y));
                raw = add(raw, mul(q[6], x3));
                raw = add(raw, mul(q[7], y3));
                raw = add(raw, mul(mul(q[8], x2), y));
                raw = add(raw, mul(mul(q[9], x), y2));
                raw = add(raw, mul(mul(q[10], x2), x2));
                raw = add(raw, mul(mul(q[11], y2), y2));
                raw = add(raw, mul(mul(q[12], x3), y));
                raw = add(raw, mul(mul(q[13], x2), y2));
                raw = add(raw, mul(mul(q[14], x), y3));
                const float n = raw / 2.0f;
                const float v = raw / std::sqrt(add(1.0f, mul(n, n)));
                f[((size_t)c * 192 + m) * 3 + ch] = ::exp2f(v);
            }
        }
    }
    return f;
}

// Compressed TC coordinates of every node (gamut.rs:259-373 compress, knee,
// ray_polygon_distance; remap_tc_lut's node chromaticities). False when a node's
// compression is unusable.
bool remap_coordinates(const float* hull_xy, const float* center, std::vector<float>& out) {
    out.assign((size_t)kNodes * 2, 0.0f);
    const double c0 = center[0], c1 = center[1];
    for (int c = 0; c < 192; ++c) {
        const float root = std::sqrt((float)c / 191.0f);
        for (int m = 0; m < 192; ++m) {
            const float xy0 = add(1.0f, -root), xy1 = mul((float)m / 191.0f, root);
            const double dx = (double)xy0 - c0, dy = (double)xy1 - c1;
            const double dist = std::hypot(dx, dy);
            float rx = xy0, ry = xy1;
            if (!(dist < 1e-9)) {
                const double ux = dx / dist, uy = dy / dist;
                double best = INFINITY;
                for (int k = 0; k < 1024; ++k) {
                    const double ax = hull_xy[2 * k], ay = hull_xy[2 * k + 1];
                    const double ex = (double)hull_xy[2 * k + 2] - ax, ey = (double)hull_xy[2 * k + 3] - ay;
                    const double den = ux * ey - uy * ex;
                    if (std::fabs(den) <= 1e-12) continue;
                    const double ox = c0 - ax, oy = c1 - ay;
                    const double d = (-ox * ey + oy * ex) / den;
                    if (d > 1e-9 && d < best) {
                        const double pos = (-ox * uy + oy * ux) / den;
                        if (pos >= -1e-9 && pos <= 1.0 + 1e-9) best = d;
                    }
                }
                if (!std::isfinite(best) || best <= 1e-12) return false;
                double t = dist / best;
                if (t > 0.815) {
                    const double scale = 1.0 - 0.815;
                    const double u = (t - 0.815) / scale;
                    t = 0.815 + scale * (u / std::pow(1.0 + std::pow(u, 1.2), 1.0 / 1.2));
                }
                const double cd = t * best;
                const double px = c0 + ux * cd, py = c1 + uy * cd;
                if (!std::isfinite(px) || !std::isfinite(py)) return false;
                rx = (float)px;
                ry = (float)py;
            }
            // tri2quad (reconstruction.rs:352-356)
            const float x = add(1.0f, -rx);
            const float dn = x < 1e-10f ? 1e-10f : x;
            out[((size_t)c * 192 + m) * 2] = std::fmin(std::fmax(mul(x, x), 0.0f), 1.0f);
            out[((size_t)c * 192 + m) * 2 + 1] = std::fmin(std::fmax(ry / dn, 0.0f), 1.0f);
        }
    }
    return true;
}

} // namespace

} // namespace fjb

extern "C" FjStatus fjb_tc_lut_build(const FjbTcLutInput* in, float* table, void* stream, FjErrorBuffer* error) {
    using namespace fjb;
    try {
        if (!in || !table || !in->spectra || !in->sensitivity_rgb || !in->reference_illuminant)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (in->method != 0 && in->method != 2)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: method must be Hanatos (0) or Arctic (2)");
        if (in->apply_surface && (in->method != 0 || !in->surface_rgb))
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error,
                               "TC LUT: the surface correction needs the Hanatos method and its 3 x 15 parameters");
        TcParams p{};
        std::memcpy(p.sens, in->sensitivity_rgb, sizeof(p.sens));
        std::memcpy(p.illum, in->reference_illuminant, sizeof(p.illum));
        for (float v : p.illum)
            if (!std::isfinite(v) || v < 0.0f)
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error,
                                   "TC LUT: requirement=finite_nonnegative_reference_illuminant");
        const float sigma = in->spectral_blur;
        if (in->method == 0 && sigma > 0.0f) {
            if (!std::isfinite(sigma)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_blur");
            const float rounded = add(mul(4.0f, sigma), 0.5f);
            if (!std::isfinite(rounded) || rounded < 1.0f)
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_blur_kernel");
            const long long radius = (long long)rounded;
            if (radius > (kMaxBlurTaps - 1) / 2)
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: spectral blur radius above 80 samples");
            const float s2 = mul(sigma, sigma);
            float sum = 0.0f;
            for (long long k = 0; k <= 2 * radius; ++k) {
                const long long off = k - radius;
                const float w = std::exp(mul(-0.5f, (float)(off * off)) / s2);
                p.taps[k] = w;
                sum = add(sum, w);
            }
            if (!std::isfinite(sum) || !(sum > 0.0f))
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_blur_kernel");
            for (long long k = 0; k <= 2 * radius; ++k) p.taps[k] = p.taps[k] / sum;
            p.radius = (int)radius;
        }
        if (in->method == 2) {
            p.arctic = 1;
            const float* w = in->projection_white_xyz;
            const float sum = add(add(w[0], w[1]), w[2]);
            if (!std::isfinite(sum) || !(sum > 0.0f))
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_d65_projection_white");
            const float tx = w[0] / sum, ty = w[1] / sum;
            const float x = add(1.0f, -tx);
            const float den = x < 1e-10f ? 1e-10f : x;
            p.tc_c = std::fmin(std::fmax(mul(x, x), 0.0f), 1.0f);
            p.tc_m = std::fmin(std::fmax(ty / den, 0.0f), 1.0f);
            if (!std::isfinite(p.tc_c) || !std::isfinite(p.tc_m))
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_d65_projection_white");
        }
        std::vector<float> factors;
        if (in->apply_surface) {
            const float* w = in->projection_white_xyz;
            const float sum = add(add(w[0], w[1]), w[2]);
            if (!std::isfinite(sum) || !(sum > 0.0f))
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error,
                                   "TC LUT: requirement=finite_surface_reference_white");
            const float tx = w[0] / sum, ty = w[1] / sum;
            const float x = add(1.0f, -tx);
            const float den = x < 1e-10f ? 1e-10f : x;
            const float cc = std::fmin(std::fmax(mul(x, x), 0.0f), 1.0f);
            const float cm = std::fmin(std::fmax(ty / den, 0.0f), 1.0f);
            if (!std::isfinite(cc) || !std::isfinite(cm))
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error,
                                   "TC LUT: requirement=finite_surface_reference_white");
            factors = surface_factors(in->surface_rgb, cc, cm);
        }
        // the compression's node coordinates (their failure is reported after the build's)
        std::vector<float> coords;
        const bool compress = in->input_compression != 0, hull = in->hull_available && in->hull_xy;
        const bool coords_ok = compress && hull && remap_coordinates(in->hull_xy, in->hull_center, coords);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        // denominators, failure flags, surface factors, the table before the remap and the
        // remap coordinates: freed before the call returns
        const size_t built_bytes = coords_ok ? (size_t)kNodes * 4 * sizeof(float) : 0;
        const size_t bytes = 256 + (factors.size() * sizeof(float) + 255) / 256 * 256 + built_bytes +
                             coords.size() * sizeof(float);
        void* scratch = nullptr;
        cudaError_t e = cudaMalloc(&scratch, bytes);
        if (e != cudaSuccess) return cuda_status(e, error, "TC LUT scratch");
        float* den = static_cast<float*>(scratch);
        unsigned* flags = reinterpret_cast<unsigned*>(den + 3);
        char* cursor = static_cast<char*>(scratch) + 256;
        float* surface = factors.empty() ? nullptr : reinterpret_cast<float*>(cursor);
        cursor += (factors.size() * sizeof(float) + 255) / 256 * 256;
        float* built = coords_ok ? reinterpret_cast<float*>(cursor) : nullptr;
        cursor += built_bytes;
        float2* tc = coords_ok ? reinterpret_cast<float2*>(cursor) : nullptr;
        e = cudaMemsetAsync(scratch, 0, 16, s);
        // pageable source: the copy completes before cudaMemcpyAsync returns
        if (e == cudaSuccess && surface)
            e = cudaMemcpyAsync(surface, factors.data(), factors.size() * sizeof(float), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && tc)
            e = cudaMemcpyAsync(tc, coords.data(), coords.size() * sizeof(float), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && p.arctic) {
            fjb::count_launch();
            tc_neutral_kernel<<<1, 1, 0, s>>>(in->spectra, p, den, flags);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            fjb::count_launch();
            tc_lut_kernel<<<(kNodes + 127) / 128, 128, 0, s>>>(in->spectra, p, den, surface, built ? built : table,
                                                               flags);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && built) {
            fjb::count_launch();
            tc_remap_kernel<<<(kNodes + 127) / 128, 128, 0, s>>>(built, tc, table, flags);
            e = cudaGetLastError();
        }
        unsigned f = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&f, flags, sizeof(f), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(scratch);
        if (e != cudaSuccess) return cuda_status(e, error, "TC LUT build");
        // the reference blurs every spectrum first, then forms the neutral response,
        // then integrates: its first failure in that order is the one reported
        if (f & kBlurNonFinite)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_blurred_spectra");
        if (f & kNeutralInvalid)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_positive_neutral_response");
        if (f & kIntegratedNonFinite)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_integrated_samples");
        if (compress && !hull)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=input_compression_hull");
        if (compress && !coords_ok)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=usable_compressed_coordinates");
        if (f & kSamplingUnusable)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=usable_sampling_coordinates");
        if (f & kRemappedNonFinite)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "TC LUT: requirement=finite_remapped_samples");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_tc_lut_build");
    }
}
