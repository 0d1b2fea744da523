// fjb_pixel_math.cuh -- per-pixel film-process math of the fused render chain.
//
// Each function restates one step of Film-Juicer's per-pixel model; the reference
// location of the same step is cited beside it. The arithmetic (operation order,
// FP32 vs FP64, sanitisation and failure rules) follows the reference so that the
// chain agrees with it to FP32 rounding; the data layout is this project's own
// (vector-packed LUT nodes, curves in shared memory, print coefficients in the
// constant bank).
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#include "fjb_params.h"

namespace fjb {

__device__ __forceinline__ bool finite_f(float v) { return isfinite(v); }
__device__ __forceinline__ float keep_finite(float v) { return isfinite(v) ? v : 0.0f; }
__device__ __forceinline__ float keep_finite_nonneg(float v) { return isfinite(v) ? fmaxf(0.0f, v) : 0.0f; }

__device__ __forceinline__ void mat3_apply(const float m[9], const float v[3], float o[3]) {
    o[0] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    o[1] = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    o[2] = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
}

__device__ __forceinline__ void mat3_apply_d(const float m[9], const double v[3], double o[3]) {
    o[0] = (double)m[0] * v[0] + (double)m[1] * v[1] + (double)m[2] * v[2];
    o[1] = (double)m[3] * v[0] + (double)m[4] * v[1] + (double)m[5] * v[2];
    o[2] = (double)m[6] * v[0] + (double)m[7] * v[1] + (double)m[8] * v[2];
}

// ---------------------------------------------------------------------------
// a1: input decoding and colour conversion
// (src/Cuda/JuicerCudaDeviceHelpers.cuh:175-231, :509-561)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float decode_srgb(float v) {
    const float x = fmaxf(0.0f, keep_finite(v));
    if (x <= 0.04045f) return x / 12.92f;
    return powf((x + 0.055f) / 1.055f, 2.4f);
}

__device__ __forceinline__ float decode_bt2020(float v) {
    const float x = fmaxf(0.0f, keep_finite(v));
    const float a = 1.09929681f;
    if (x < 0.0812428791f) return x / 4.5f;
    return powf((x + (a - 1.0f)) / a, 1.0f / 0.45f);
}

__device__ __forceinline__ void decode_input(const PixelParams& p, const float in[3], float lin[3]) {
    if (p.decode_cctf && p.input_color_space == 1) {
        for (int c = 0; c < 3; ++c) lin[c] = decode_bt2020(in[c]);
    } else if (p.decode_cctf && p.input_color_space == 3) {
        for (int c = 0; c < 3; ++c) lin[c] = decode_srgb(in[c]);
    } else {
        for (int c = 0; c < 3; ++c) lin[c] = keep_finite(in[c]);
    }
}

// ---------------------------------------------------------------------------
// a2: Hanatos / Arctic exposure through the 192x192 TC LUT with 4x4 Mitchell taps
// (src/Cuda/JuicerCudaDeviceHelpers.cuh:233-327, :563-617)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float mitchell(float t) {
    const float B = 1.0f / 3.0f;
    const float C = 1.0f / 3.0f;
    const float x = fabsf(t);
    if (x < 1.0f) {
        return (1.0f / 6.0f) * ((12.0f - 9.0f * B - 6.0f * C) * x * x * x +
                                (-18.0f + 12.0f * B + 6.0f * C) * x * x + (6.0f - 2.0f * B));
    }
    if (x < 2.0f) {
        return (1.0f / 6.0f) * ((-B - 6.0f * C) * x * x * x + (6.0f * B + 30.0f * C) * x * x +
                                (-12.0f * B - 48.0f * C) * x + (8.0f * B + 24.0f * C));
    }
    return 0.0f;
}

__device__ __forceinline__ void tc_coordinate(float normalized, int& base, float& frac) {
    const float top = (float)(kTcLutExtent - 1);
    const float coord = fminf(1.0f, fmaxf(0.0f, normalized)) * top;
    if (coord >= top) {
        base = kTcLutExtent - 2;
        frac = 1.0f;
        return;
    }
    base = (int)floorf(coord);
    frac = coord - (float)base;
}

__device__ __forceinline__ int tc_reflect(int i) {
    if (i < 0) return -i;
    if (i >= kTcLutExtent) return 2 * (kTcLutExtent - 1) - i;
    return i;
}

// Footprints that touch the LUT border reflect their indices (cold path, out of line).
static __device__ __noinline__ void tc_lut_edge(const float4* __restrict__ lut, int cb, int mb, float cf, float mf,
                                         float acc[3], float& wsum) {
    const float wc[4] = {mitchell(cf + 1.0f), mitchell(cf), mitchell(cf - 1.0f), mitchell(cf - 2.0f)};
    const float wm[4] = {mitchell(mf + 1.0f), mitchell(mf), mitchell(mf - 1.0f), mitchell(mf - 2.0f)};
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, ws = 0.0f;
#pragma unroll
    for (int dc = 0; dc < 4; ++dc) {
        const int c = tc_reflect(cb - 1 + dc);
#pragma unroll
        for (int dm = 0; dm < 4; ++dm) {
            const int m = tc_reflect(mb - 1 + dm);
            const float w = wc[dc] * wm[dm];
            ws += w;
            const float4 t = __ldg(lut + c * kTcLutExtent + m);
            a0 += w * t.x;
            a1 += w * t.y;
            a2 += w * t.z;
        }
    }
    acc[0] = a0;
    acc[1] = a1;
    acc[2] = a2;
    wsum = ws;
}

// All three channels of one tap come from one 16-byte load.
__device__ __forceinline__ void tc_lut_sample(const float4* __restrict__ lut, float qx, float qy, float rgb[3]) {
    int cb, mb;
    float cf, mf;
    tc_coordinate(qx, cb, cf);
    tc_coordinate(qy, mb, mf);
    const float wc[4] = {mitchell(cf + 1.0f), mitchell(cf), mitchell(cf - 1.0f), mitchell(cf - 2.0f)};
    const float wm[4] = {mitchell(mf + 1.0f), mitchell(mf), mitchell(mf - 1.0f), mitchell(mf - 2.0f)};
    float acc[3] = {0.0f, 0.0f, 0.0f};
    float wsum = 0.0f;
    if (cb >= 1 && cb <= kTcLutExtent - 3 && mb >= 1 && mb <= kTcLutExtent - 3) {
        // Interior cell: the 4x4 footprint needs no reflection; one base pointer with
        // compile-time offsets.
        const float4* base = lut + (cb - 1) * kTcLutExtent + (mb - 1);
#pragma unroll
        for (int dc = 0; dc < 4; ++dc) {
#pragma unroll
            for (int dm = 0; dm < 4; ++dm) {
                const float w = wc[dc] * wm[dm];
                wsum += w;
                const float4 t = __ldg(base + dc * kTcLutExtent + dm);
                acc[0] += w * t.x;
                acc[1] += w * t.y;
                acc[2] += w * t.z;
            }
        }
    } else {
        tc_lut_edge(lut, cb, mb, cf, mf, acc, wsum);
    }
    for (int k = 0; k < 3; ++k) rgb[k] = wsum != 0.0f ? acc[k] / wsum : 0.0f;
}

__device__ __forceinline__ void working_xyz(const PixelParams& p, const float in[3], float xyz[3]) {
    float lin[3], raw[3];
    decode_input(p, in, lin);
    mat3_apply(p.input_rgb_to_xyz, lin, raw);
    if (p.adapt_input) {
        mat3_apply(p.input_xyz_adapt, raw, xyz);
    } else {
        xyz[0] = raw[0];
        xyz[1] = raw[1];
        xyz[2] = raw[2];
    }
    for (int c = 0; c < 3; ++c) xyz[c] = keep_finite(xyz[c]);
}

__device__ __forceinline__ void tc_exposure(const PixelParams& p, const float in_xyz[3], float e_bgr[3]) {
    const float X = keep_finite(in_xyz[0]);
    const float Y = keep_finite(in_xyz[1]);
    const float Z = keep_finite(in_xyz[2]);
    const float sum = X + Y + Z;
    const float den = fmaxf(sum, 1e-10f);
    const float tx = X / den;
    const float ty = Y / den;
    // triangle -> square mapping of chromaticity
    const float one_minus = 1.0f - tx;
    const float qden = fmaxf(one_minus, 1e-10f);
    const float qx = fminf(1.0f, fmaxf(0.0f, one_minus * one_minus));
    const float qy = fminf(1.0f, fmaxf(0.0f, ty / qden));
    float rgb[3];
    tc_lut_sample(p.tc_lut, qx, qy, rgb);
    e_bgr[0] = keep_finite(sum * keep_finite(rgb[2]));
    e_bgr[1] = keep_finite(sum * keep_finite(rgb[1]));
    e_bgr[2] = keep_finite(sum * keep_finite(rgb[0]));
}

// ---------------------------------------------------------------------------
// a3: Mallett 2019 81-lambda basis exposure (src/Cuda/JuicerCudaDeviceHelpers.cuh:619-668)
// ---------------------------------------------------------------------------
static __device__ __noinline__ void mallett_exposure(const PixelParams& p, const float in[3], float e_bgr[3]) {
    float lin[3], xyz[3], ad[3], srgb[3];
    decode_input(p, in, lin);
    mat3_apply(p.input_rgb_to_xyz, lin, xyz);
    const float* src = xyz;
    if (p.adapt_input) {
        mat3_apply(p.input_xyz_adapt, xyz, ad);
        src = ad;
    }
    mat3_apply(p.xyz_to_linear_srgb, src, srgb);
    const float r = fmaxf(0.0f, keep_finite(keep_finite(srgb[0])));
    const float g = fmaxf(0.0f, keep_finite(keep_finite(srgb[1])));
    const float b = fmaxf(0.0f, keep_finite(keep_finite(srgb[2])));
    float eb = 0.0f, eg = 0.0f, er = 0.0f;
    const float* sb = p.film_sens_bgr;
    const float* sg = p.film_sens_bgr + kSpectralSamples;
    const float* sr = p.film_sens_bgr + 2 * kSpectralSamples;
    for (int i = 0; i < kSpectralSamples; ++i) {
        const float il = __ldg(p.mallett_illum + i);
        const float b0 = __ldg(p.mallett_basis + 3 * i);
        const float b1 = __ldg(p.mallett_basis + 3 * i + 1);
        const float b2 = __ldg(p.mallett_basis + 3 * i + 2);
        const float spd = (r * b0 + g * b1 + b * b2) * il;
        if (!finite_f(spd)) continue;
        const float vb = __ldg(sb + i), vg = __ldg(sg + i), vr = __ldg(sr + i);
        if (isfinite(vb)) eb += spd * vb;
        if (isfinite(vg)) eg += spd * vg;
        if (isfinite(vr)) er += spd * vr;
    }
    e_bgr[0] = finite_f(eb) ? fmaxf(0.0f, eb) : 0.0f;
    e_bgr[1] = finite_f(eg) ? fmaxf(0.0f, eg) : 0.0f;
    e_bgr[2] = finite_f(er) ? fmaxf(0.0f, er) : 0.0f;
    for (int c = 0; c < 3; ++c) e_bgr[c] = fmaxf(0.0f, e_bgr[c] * p.mallett_midgray_scale);
}

// a4: film linear exposure with auto, manual and route scales
// (src/Cuda/JuicerCudaDeviceHelpers.cuh:710-736)
__device__ __forceinline__ float exposure_scale(const PixelParams& p, bool with_route) {
    float ae = 1.0f;
    if (p.auto_exposure_scale) {
        const float s = *p.auto_exposure_scale;
        if (isfinite(s) && s > 0.0f) ae = s;
    }
    float scale = ae * p.manual_exposure_scale;
    if (with_route) scale *= p.route_correction_scale;
    return (isfinite(scale) && scale > 0.0f) ? scale : 1.0f;
}

__device__ __forceinline__ void camera_linear_exposure(const PixelParams& p, const float in[3], bool with_route,
                                                       float e_bgr[3]) {
    if (p.method == kMallett) {
        mallett_exposure(p, in, e_bgr);
    } else {
        float xyz[3];
        working_xyz(p, in, xyz);
        tc_exposure(p, xyz, e_bgr);
    }
    const float s = exposure_scale(p, with_route);
    for (int c = 0; c < 3; ++c) e_bgr[c] = fmaxf(0.0f, e_bgr[c] * s);
}

// ---------------------------------------------------------------------------
// a5: log exposure and density-curve lookup (src/Cuda/JuicerCudaDeviceHelpers.cuh:34-105, :766-775)
// Curves live in shared memory; the interval search is the same "first abscissa
// strictly above the query" rule as the reference, so the chosen interval index is
// identical for identical queries.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float log_exposure(float e) { return log10f(fmaxf(e, 0.0f) + 1e-10f); }

// First index i1 in [1, last] with xq < x[i1] (last + 1 when none): the reference's
// binary search (src/Cuda/JuicerCudaDeviceHelpers.cuh:59-71).
static __device__ __noinline__ int curve_interval_search(const float* x, int last, float xq) {
    int lo = 1, hi = last, i1 = last + 1;
    while (lo <= hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (xq < x[mid]) {
            i1 = mid;
            hi = mid - 1;
        } else {
            lo = mid + 1;
        }
    }
    return i1;
}

__device__ __forceinline__ float curve_sample(const float* __restrict__ blob, const CurveRef& c, float logE,
                                              float gamma) {
    if (!isfinite(logE)) return nanf("");
    const float* x = blob + c.x;
    const float* y = blob + c.y;
    const int last = c.n - 1;
    const float xq = logE * gamma;
    const float xmin = x[0];
    const float xmax = x[last];
    if (!(xmax >= xmin)) return y[0];
    if (xq <= xmin) return y[0];
    if (xq >= xmax) return y[last];
    int i1 = last + 1;
    bool found = false;
    if (c.guess) {
        // Strictly increasing, near-uniform abscissa: start from the uniform-grid cell
        // and step to the unique i1 with x[i1-1] <= xq < x[i1] (the interval the
        // reference's binary search selects). Two steps either way cover the spacing
        // jitter the host admitted; otherwise fall through to the binary search.
        int g = (int)((xq - c.x0) * c.inv_dx);
        g = g < 0 ? 0 : (g > last - 1 ? last - 1 : g);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (g > 0 && xq < x[g]) --g;
            if (g < last - 1 && xq >= x[g + 1]) ++g;
        }
        if (x[g] <= xq && xq < x[g + 1]) {
            i1 = g + 1;
            found = true;
        }
    }
    if (!found) i1 = curve_interval_search(x, last, xq);
    if (i1 > last) return y[last];
    const int i0 = i1 - 1;
    const float x0 = x[i0], x1 = x[i1], y0 = y[i0], y1 = y[i1];
    const float den = x1 - x0;
    if (!(den > 0.0f) || !isfinite(den)) return y0;
    const float t = (xq - x0) / den;
    return y0 + t * (y1 - y0);
}

__device__ __forceinline__ float clamp_infinite_log(const float* __restrict__ blob, CurveRef c, float logE) {
    if (isfinite(logE) || isnan(logE)) return logE;
    const float xmin = blob[c.x];
    const float xmax = blob[c.x + c.n - 1];
    if (!(xmax >= xmin)) return logE;
    return logE > 0.0f ? xmax : xmin;
}

// ---------------------------------------------------------------------------
// a6: DIR coupler chemistry (src/Cuda/JuicerCudaDeviceHelpers.cuh:1073-1265)
// ---------------------------------------------------------------------------
// Overflow-safe evaluation of the Langmuir term when the direct product could
// overflow or hit the receiver pole (cold path, kept out of line).
static __device__ __noinline__ bool langmuir_guarded(float value, float knee, float ref, float den, float& out) {
    const float num_scale = 1.0f + ref / knee;
    if (!isfinite(num_scale)) return false;
    if (value >= 0.0f) {
        const float den_scale = 1.0f + value / knee;
        if (!isfinite(den_scale) || den_scale == 0.0f) return false;
        out = (value / den_scale) * num_scale;
        return isfinite(out);
    }
    if (!isfinite(den) || den == 0.0f) return false;
    const float den_scale = den / knee;
    if (!isfinite(den_scale) || den_scale == 0.0f) return false;
    if (fabsf(value) <= FLT_MAX / fabsf(num_scale)) {
        out = value * num_scale / den_scale;
    } else {
        out = (value / den_scale) * num_scale;
    }
    return isfinite(out);
}

__device__ __forceinline__ bool langmuir(float value, float knee, float ref, float& out) {
    out = nanf("");
    if (!isfinite(value) || !isfinite(knee) || !(knee > 0.0f) || !isfinite(ref)) return false;
    const float den = knee + value;
    const float kr = knee + ref;
    const bool direct = isfinite(den) && den != 0.0f && isfinite(kr) &&
                        (value == 0.0f || fabsf(value) <= FLT_MAX / fabsf(kr));
    if (direct) {
        out = value * kr / den;
        return isfinite(out);
    }
    return langmuir_guarded(value, knee, ref, den, out);
}

// Donor corrections for layer densities (B, G, R); returns a channel failure mask.
__device__ __forceinline__ unsigned dir_donor_corrections(const PixelParams& p, const float layer[3], float corr[3]) {
    if (p.dir_mode == kDirInactive) {
        corr[0] = corr[1] = corr[2] = 0.0f;
        return 0u;
    }
    float donor[3] = {p.dir_dmax[0] - layer[0], p.dir_dmax[1] - layer[1], p.dir_dmax[2] - layer[2]};
    unsigned fail = 0u;
    if (p.dir_mode == kDirNegativeDonor) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (!langmuir(layer[c], p.dir_donor_k[c], p.dir_dref[c], donor[c])) fail |= 1u << c;
        }
    }
    const float* M = p.dir_m;
    corr[0] = M[0] * donor[0] + M[3] * donor[1] + M[6] * donor[2];
    corr[1] = M[1] * donor[0] + M[4] * donor[1] + M[7] * donor[2];
    corr[2] = M[2] * donor[0] + M[5] * donor[1] + M[8] * donor[2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        if (!isfinite(corr[c])) fail |= 1u << c;
    return fail;
}

__device__ __forceinline__ unsigned dir_receiver_finalize(const PixelParams& p, float corr[3]) {
    if (p.dir_mode != kDirPositiveReceiver) return 0u;
    unsigned fail = 0u;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (p.dir_receiver_cref[c] == 0.0f) {
            corr[c] = 0.0f;
            continue;
        }
        const float v = corr[c];
        if (!langmuir(v, p.dir_receiver_kr[c], p.dir_receiver_cref[c], corr[c])) fail |= 1u << c;
    }
    return fail;
}

// Subtracts corrections from log exposure, flagging channels whose result stops being
// a consistent number (the reference's signed-infinity rule).
__device__ __forceinline__ unsigned subtract_corrections(const float logE[3], const float corr[3], float out[3]) {
    unsigned fail = 0u;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float o = logE[c];
        if (isnan(o)) {
            fail |= 1u << c;
            out[c] = 0.0f;
            continue;
        }
        out[c] = o - corr[c];
        if ((!isinf(o) && !isfinite(out[c])) ||
            (isinf(o) && (!isinf(out[c]) || signbit(o) != signbit(out[c])))) {
            fail |= 1u << c;
        }
    }
    return fail;
}

__device__ __forceinline__ void flag_dir_failure(const PixelParams& p, unsigned mask) {
    if (p.error_flags && mask != 0u) atomicOr(p.error_flags, (1u << 8) | ((mask & 7u) << 9));
}

__device__ __forceinline__ void flag_scan_failure(const PixelParams& p) {
    if (p.error_flags) atomicOr(p.error_flags, 1u);
}

// Capture development from film linear exposure (B, G, R) to dye density (C, M, Y).
// Runtime DIR (src/Cuda/Scan/JuicerCudaScanPipeline.cu:1622-1698 with
// src/Cuda/JuicerCudaDeviceHelpers.cuh:833-846, :1206-1241).
__device__ __forceinline__ void develop_capture(const PixelParams& p, const float* __restrict__ blob,
                                                const float e_bgr[3], float dens_cmy[3]) {
    float logE[3], logS[3], layer[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        logE[c] = log_exposure(e_bgr[c]);
        logS[c] = clamp_infinite_log(blob, p.film_curve[c], logE[c]);
        layer[c] = curve_sample(blob, p.film_curve[c], logS[c], p.gamma_bgr[c]);
    }
    if (p.dir_mode == kDirInactive) {
        dens_cmy[0] = layer[2];
        dens_cmy[1] = layer[1];
        dens_cmy[2] = layer[0];
        return;
    }
    float corr[3];
    unsigned fail = dir_donor_corrections(p, layer, corr);
    fail |= dir_receiver_finalize(p, corr);
    float logC[3];
    if (fail == 0u) fail = subtract_corrections(logS, corr, logC);
    if (fail != 0u) {
        flag_dir_failure(p, fail);
        dens_cmy[0] = dens_cmy[1] = dens_cmy[2] = nanf("");
        return;
    }
    dens_cmy[2] = curve_sample(blob, p.dir_curve[0], logC[0], p.gamma_bgr[0]);
    dens_cmy[1] = curve_sample(blob, p.dir_curve[1], logC[1], p.gamma_bgr[1]);
    dens_cmy[0] = curve_sample(blob, p.dir_curve[2], logC[2], p.gamma_bgr[2]);
}

// Capture development with spatially filtered DIR corrections
// (src/Cuda/JuicerCudaDeviceHelpers.cuh:1267-1328).
__device__ __forceinline__ void develop_capture_spatial(const PixelParams& p, const float* __restrict__ blob,
                                                        const float logRaw[3], float corr_in[3],
                                                        float dens_cmy[3]) {
    float corr[3] = {corr_in[0], corr_in[1], corr_in[2]};
    unsigned fail = dir_receiver_finalize(p, corr);
    float logC[3];
    if (fail == 0u) fail = subtract_corrections(logRaw, corr, logC);
    if (fail != 0u) {
        flag_dir_failure(p, fail);
        dens_cmy[0] = dens_cmy[1] = dens_cmy[2] = nanf("");
        return;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) logC[c] = clamp_infinite_log(blob, p.film_curve[c], logC[c]);
    dens_cmy[2] = curve_sample(blob, p.dir_curve[0], logC[0], p.gamma_bgr[0]);
    dens_cmy[1] = curve_sample(blob, p.dir_curve[1], logC[1], p.gamma_bgr[1]);
    dens_cmy[0] = curve_sample(blob, p.dir_curve[2], logC[2], p.gamma_bgr[2]);
}

// ---------------------------------------------------------------------------
// a8: enlarger print exposure + development (src/Cuda/JuicerCudaDeviceHelpers.cuh:860-1071)
// The 81-wavelength coefficients are read straight from the constant bank.
// ---------------------------------------------------------------------------
// 2^x on the MUFU (ex2.approx.ftz.f32: relative error about 2^-22, flushes subnormal
// results to zero; transmittances here are >= 2^-40, far above the subnormal range).
__device__ __forceinline__ float mufu_exp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Non-finite density (a failed DIR pixel): the reference's per-sample NaN rule
// (src/Cuda/JuicerCudaDeviceHelpers.cuh:856-864). Cold path, out of line.
static __device__ __noinline__ void print_spectral_nonfinite(const PrintSpectral& s, const float d[3], float raw[3]) {
    float ac = 0.0f, am = 0.0f, ay = 0.0f;
    for (int i = 0; i < s.count; ++i) {
        const float dl = d[0] * s.nd[i][0] + d[1] * s.nd[i][1] + d[2] * s.nd[i][2] + s.nd[i][3];
        float t = exp2f(dl);
        t = isnan(t) ? 0.0f : t;
        ac += t * s.sens[i][0];
        am += t * s.sens[i][1];
        ay += t * s.sens[i][2];
    }
    raw[0] = ac;
    raw[1] = am;
    raw[2] = ay;
}

__device__ __forceinline__ void print_spectral(const PrintSpectral& s, const float d[3], float raw[3]) {
    if (isfinite(d[0]) && isfinite(d[1]) && isfinite(d[2])) {
        // Fast path: all 81 slots unrolled, coefficients are constant-bank operands
        // (one per instruction: the film base sits in the weights, fjb_params.h).
        // Finite densities give finite exponents, so no NaN guard is needed; padded
        // slots evaluate 2^0 * 0 = +0. Two partial sums per channel (even / odd
        // wavelength) halve the dependent FMA chain.
        float a0[3] = {0.0f, 0.0f, 0.0f}, a1[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int i = 0; i < kSpectralSamples; ++i) {
            const float dl = fmaf(d[0], s.nd[i][0], fmaf(d[1], s.nd[i][1], d[2] * s.nd[i][2]));
            const float t = mufu_exp2(dl);
            float* a = (i & 1) ? a1 : a0;
            a[0] = fmaf(t, s.sens[i][0], a[0]);
            a[1] = fmaf(t, s.sens[i][1], a[1]);
            a[2] = fmaf(t, s.sens[i][2], a[2]);
        }
        const float ac = a0[0] + a1[0], am = a0[1] + a1[1], ay = a0[2] + a1[2];
        raw[0] = ac;
        raw[1] = am;
        raw[2] = ay;
    } else {
        print_spectral_nonfinite(s, d, raw);
    }
}

// Print exposure from the spectral integral `raw` (C, M, Y) to print density in `d`:
// dust, mid-grey normaliser, preflash, print exposure, route correction, log10 and
// the print curves (src/Cuda/JuicerCudaDeviceHelpers.cuh:935-1071). `dust`: film
// dust transmittance of the pixel (:1062-1066).
__device__ __forceinline__ void print_finish(const PixelParams& p, const float* __restrict__ blob, float raw[3],
                                             float d[3], float dust) {
    if (dust != 1.0f)
        for (int c = 0; c < 3; ++c) raw[c] *= dust;
    const float k = p.print_midgray;
    for (int c = 0; c < 3; ++c) raw[c] *= k;
    const float pf = p.print_preflash_exposure;
    if (isfinite(pf) && pf > 0.0f) {
        for (int c = 0; c < 3; ++c) raw[c] += p.print_preflash_raw[c] * pf;
    }
    for (int c = 0; c < 3; ++c) raw[c] *= p.print_exposure;
    for (int c = 0; c < 3; ++c) raw[c] *= p.print_route_correction;
    for (int c = 0; c < 3; ++c) {
        const float lp = log10f(raw[c] + 1e-10f);
        d[c] = curve_sample(blob, p.print_curve[c], lp, 1.0f);
    }
}

// Print-linear exposure for the enlarger diffusion (src/Cuda/JuicerCudaDeviceHelpers.cuh:966-1010
// print_inner_raw_device + print_linear_for_diffusion_device): the spectral integral times
// the dust transmittance and the mid-grey normaliser, plus preflash, then
// (max(raw, 0) + 1e-10) times print exposure x route correction.
__device__ __forceinline__ void enlarger_linear(const PixelParams& p, float raw[3], float dust, float lin[3]) {
    if (dust != 1.0f)
        for (int c = 0; c < 3; ++c) raw[c] *= dust;
    for (int c = 0; c < 3; ++c) raw[c] *= p.print_midgray;
    if (p.print_preflash_exposure > 0.0f)
        for (int c = 0; c < 3; ++c) raw[c] += p.print_preflash_raw[c] * p.print_preflash_exposure;
    const float outer = p.print_exposure * p.print_route_correction;
    for (int c = 0; c < 3; ++c) lin[c] = (fmaxf(raw[c], 0.0f) + 1e-10f) * outer;
}

__device__ __forceinline__ void print_develop(const PixelParams& p, const float* __restrict__ blob, float d[3],
                                              float dust = 1.0f) {
    float raw[3];
    print_spectral(p.spectral, d, raw);
    print_finish(p, blob, raw, d, dust);
}

// ---------------------------------------------------------------------------
// a9: scanner PCHIP LUT (src/Cuda/JuicerCudaDeviceHelpers.cuh:330-506)
// Nodes are packed as (value, slope_c, slope_m, slope_y) per output so each corner
// of the cell is one 16-byte load per output.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pchip_coordinate(float normalized, int res, int& base, float& frac) {
    const float top = (float)(res - 1);
    float coord = normalized * top;
    coord = fminf(top, fmaxf(0.0f, coord));
    if (coord >= top) {
        base = res - 2;
        frac = 1.0f;
        return;
    }
    base = (int)floorf(coord);
    frac = coord - (float)base;
}

__device__ __forceinline__ float hermite(float y0, float y1, float m0, float m1, float t) {
    const float t2 = t * t;
    const float t3 = t2 * t;
    const float h00 = 2.0f * t3 - 3.0f * t2 + 1.0f;
    const float h10 = t3 - 2.0f * t2 + t;
    const float h01 = -2.0f * t3 + 3.0f * t2;
    const float h11 = t3 - t2;
    return h00 * y0 + h10 * m0 + h01 * y1 + h11 * m1;
}

__device__ __forceinline__ float lerp_ref(float a, float b, float t) { return a + t * (b - a); }

__device__ __forceinline__ bool scan_lut_sample(const PixelParams& p, const double n[3], float out[3]) {
    if (!isfinite(n[0]) || !isfinite(n[1]) || !isfinite(n[2]) || p.scan_res < 2) return false;
    const int r = p.scan_res;
    int c, m, y;
    float tc, tm, ty;
    pchip_coordinate((float)n[0], r, c, tc);
    pchip_coordinate((float)n[1], r, m, tm);
    pchip_coordinate((float)n[2], r, y, ty);
    const int s = r - 1;
    const float4* cell = p.scan_cells + 2 * ((c * s + m) * s + y);
    const float4 cmin = __ldg(cell);
    const float4 cmax = __ldg(cell + 1);
    const float lo[3] = {cmin.x, cmin.y, cmin.z};
    const float hi[3] = {cmin.w, cmax.x, cmax.y};
    // node index of corner (dc, dm, dy)
    const int n000 = (c * r + m) * r + y;
    const int sc = r * r; // stride of c
    const int sm = r;     // stride of m
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        const float4 a000 = __ldg(p.scan_nodes + 3 * (n000) + o);
        const float4 a100 = __ldg(p.scan_nodes + 3 * (n000 + sc) + o);
        const float4 a010 = __ldg(p.scan_nodes + 3 * (n000 + sm) + o);
        const float4 a110 = __ldg(p.scan_nodes + 3 * (n000 + sc + sm) + o);
        const float4 a001 = __ldg(p.scan_nodes + 3 * (n000 + 1) + o);
        const float4 a101 = __ldg(p.scan_nodes + 3 * (n000 + sc + 1) + o);
        const float4 a011 = __ldg(p.scan_nodes + 3 * (n000 + sm + 1) + o);
        const float4 a111 = __ldg(p.scan_nodes + 3 * (n000 + sc + sm + 1) + o);
        const float v000 = hermite(a000.x, a100.x, a000.y, a100.y, tc);
        const float v010 = hermite(a010.x, a110.x, a010.y, a110.y, tc);
        const float v001 = hermite(a001.x, a101.x, a001.y, a101.y, tc);
        const float v011 = hermite(a011.x, a111.x, a011.y, a111.y, tc);
        const float sm00 = lerp_ref(a000.z, a100.z, tc);
        const float sm10 = lerp_ref(a010.z, a110.z, tc);
        const float sm01 = lerp_ref(a001.z, a101.z, tc);
        const float sm11 = lerp_ref(a011.z, a111.z, tc);
        const float vy0 = hermite(v000, v010, sm00, sm10, tm);
        const float vy1 = hermite(v001, v011, sm01, sm11, tm);
        const float sy0 = lerp_ref(lerp_ref(a000.w, a100.w, tc), lerp_ref(a010.w, a110.w, tc), tm);
        const float sy1 = lerp_ref(lerp_ref(a001.w, a101.w, tc), lerp_ref(a011.w, a111.w, tc), tm);
        const float v = hermite(vy0, vy1, sy0, sy1, ty);
        out[o] = fminf(hi[o], fmaxf(lo[o], v));
    }
    return true;
}

// ---------------------------------------------------------------------------
// a11: OkLch output gamut compression (src/GamutCompression.h:110-216)
// ---------------------------------------------------------------------------
__device__ __constant__ const float kOkXyzToLms[9] = {0.8189330101f, 0.3618667424f, -0.1288597137f,
                                                      0.0329845436f, 0.9293118715f, 0.0361456387f,
                                                      0.0482003018f, 0.2643662691f, 0.6338517070f};
__device__ __constant__ const float kOkLmsToXyz[9] = {1.2270138511f,  -0.5577999807f, 0.2812561490f,
                                                      -0.0405801784f, 1.1122568696f,  -0.0716766787f,
                                                      -0.0763812845f, -0.4214819784f, 1.5861632204f};
__device__ __constant__ const float kOkLmsRootToLab[9] = {0.2104542553f, 0.7936177850f,  -0.0040720468f,
                                                          1.9779984951f, -2.4285922050f, 0.4505937099f,
                                                          0.0259040371f, 0.7827717662f,  -0.8086757660f};
__device__ __constant__ const float kOkLabToLmsRoot[9] = {1.0f, 0.3963377774f,  0.2158037573f,
                                                          1.0f, -0.1055613458f, -0.0638541728f,
                                                          1.0f, -0.0894841775f, -1.2914855480f};

__device__ __forceinline__ float signed_cbrt(float v) { return v < 0.0f ? -cbrtf(-v) : cbrtf(v); }

__device__ __forceinline__ float reinhard_knee(float v, const float knee[3]) {
    if (!(v > knee[0])) return v;
    const float span = knee[1] - knee[0];
    const float nrm = (v - knee[0]) / span;
    return knee[0] + span * nrm / powf(1.0f + powf(nrm, knee[2]), 1.0f / knee[2]);
}

__device__ __forceinline__ float gamut_boundary(const float* __restrict__ cmax, float L, float h) {
    const float kPi = 3.14159265358979323846f;
    const float kTwoPi = 2.0f * kPi;
    const float Lc = fminf(fmaxf(L, 0.02f), 1.0f);
    const float lp = (Lc - 0.02f) / (1.0f - 0.02f) * (float)(kGamutLightness - 1);
    const int l0 = (int)floorf(lp);
    const int l1 = l0 + 1 < kGamutLightness ? l0 + 1 : l0;
    const float lf = lp - (float)l0;
    float wh = fmodf(h + kPi, kTwoPi);
    if (wh < 0.0f) wh += kTwoPi;
    const float hp = wh / kTwoPi * (float)kGamutHue;
    const int h0 = (int)floorf(hp) % kGamutHue;
    const int h1 = (h0 + 1) % kGamutHue;
    const float hf = hp - floorf(hp);
    const int r0 = l0 * kGamutHue, r1 = l1 * kGamutHue;
    const float c00 = __ldg(cmax + r0 + h0), c01 = __ldg(cmax + r0 + h1);
    const float c10 = __ldg(cmax + r1 + h0), c11 = __ldg(cmax + r1 + h1);
    const float first = c00 + hf * (c01 - c00);
    const float second = c10 + hf * (c11 - c10);
    return first + lf * (second - first);
}

__device__ __forceinline__ void gamut_compress(const PixelParams& p, float rgb[3]) {
    float xyz[3], lms[3], lab[3];
    mat3_apply(p.gamut_native_to_xyz, rgb, xyz);
    mat3_apply(kOkXyzToLms, xyz, lms);
    for (int c = 0; c < 3; ++c) lms[c] = signed_cbrt(lms[c]);
    mat3_apply(kOkLmsRootToLab, lms, lab);
    lab[0] = reinhard_knee(lab[0], p.gamut_lightness_knee);
    const float chroma = hypotf(lab[1], lab[2]);
    if (chroma > 0.0f) {
        const float hue = atan2f(lab[2], lab[1]);
        const float bound = fmaxf(gamut_boundary(p.gamut_cmax, lab[0], hue), 1.0e-9f);
        const float comp = reinhard_knee(chroma / bound, p.gamut_chroma_knee) * bound;
        const float sc = comp / chroma;
        lab[1] *= sc;
        lab[2] *= sc;
    }
    mat3_apply(kOkLabToLmsRoot, lab, lms);
    for (int c = 0; c < 3; ++c) lms[c] = lms[c] * lms[c] * lms[c];
    mat3_apply(kOkLmsToXyz, lms, xyz);
    mat3_apply(p.gamut_xyz_to_native, xyz, rgb);
}

// ---------------------------------------------------------------------------
// a12: output encoding (src/Cuda/Scan/JuicerCudaScanPipeline.cu:99-192)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double clamp01(double v) {
    if (v <= 0.0) return 0.0;
    if (v >= 1.0) return 1.0;
    return v;
}

static __device__ __noinline__ float encode_channel_other(const PixelParams& p, float v);

__device__ __forceinline__ float encode_channel(const PixelParams& p, float v) {
    if (p.cctf_kind == 2) {
        if (v <= 0.0031308f) return 12.92f * v;
        return 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
    }
    return encode_channel_other(p, v);
}

// The other transfer functions, out of line to keep the hot kernel's code small.
static __device__ __noinline__ float encode_channel_other(const PixelParams& p, float v) {
    switch (p.cctf_kind) {
        case 0:
            return v;
        case 1:
            return copysignf(powf(fabsf(v), p.cctf_gamma), v);
        case 2:
            if (v <= 0.0031308f) return 12.92f * v;
            return 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
        case 3:
            if (v < p.cctf_b) return v * 4.5f;
            return p.cctf_a * powf(v, 0.45f) - (p.cctf_a - 1.0f);
        case 4:
            if (v < p.cctf_linear_cutoff) return v * 16.0f;
            return powf(v, p.cctf_gamma);
        case 5: {
            const float lin = fmaxf(0.0f, v);
            if (lin <= p.cctf_linear_cutoff) return lin * p.cctf_d;
            return (log2f(lin + p.cctf_a) + p.cctf_b) * p.cctf_c;
        }
        default:
            return (float)clamp01(v);
    }
}

__device__ __forceinline__ void encode_output(const PixelParams& p, double rgb[3]) {
    double lin[3];
    if (p.encode_input_is_output) {
        lin[0] = rgb[0];
        lin[1] = rgb[1];
        lin[2] = rgb[2];
    } else {
        mat3_apply_d(p.encode_dwg_to_output, rgb, lin);
    }
    if (p.encode_apply_cctf) {
        for (int c = 0; c < 3; ++c) rgb[c] = encode_channel(p, (float)lin[c]);
    } else {
        for (int c = 0; c < 3; ++c) rgb[c] = lin[c];
    }
    for (int c = 0; c < 3; ++c) rgb[c] = clamp01(rgb[c]);
}

// ---------------------------------------------------------------------------
// a9-a12 combined: density (C, M, Y) -> encoded output RGB. Returns false on a scan
// failure (the pixel is then written as black).
// (src/Cuda/Scan/JuicerCudaScanPipeline.cu:1757-1858)
// ---------------------------------------------------------------------------
// glare: the scanner-glare percent of the pixel, or a negative value for none.
// dust: film dust transmittance of the pixel, when the direct route scans a frame with
// film defects (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2006-2011).
__device__ __forceinline__ bool scan_to_linear(const PixelParams& p, const float d[3], double rgb[3],
                                               float glare_percent = -1.0f, const float* dust = nullptr) {
    double nd[3];
    for (int c = 0; c < 3; ++c) {
        if (p.scan_medium_negative) {
            nd[c] = ((double)d[c] + (double)p.scan_min_cmy[c]) * (double)p.scan_inv_span_cmy[c];
        } else {
            nd[c] = ((double)d[c] - (double)p.scan_min_cmy[c]) * (double)p.scan_inv_span_cmy[c];
        }
    }
    float l2[3];
    if (!scan_lut_sample(p, nd, l2)) return false;
    double xyz[3] = {(double)exp2f(l2[0]), (double)exp2f(l2[1]), (double)exp2f(l2[2])};
    if (dust) {
        const double t = *dust;
        xyz[0] *= t;
        xyz[1] *= t;
        xyz[2] *= t;
    }
    if (p.correction_active) {
        const double cy = fmin(fmax((double)p.correction_slope * xyz[1] + (double)p.correction_offset, 0.0), 1.0);
        const double sc = cy / (xyz[1] + 1e-10);
        xyz[0] *= sc;
        xyz[1] *= sc;
        xyz[2] *= sc;
    }
    if (glare_percent >= 0.0f) {
        // src/Cuda/Scan/JuicerCudaScanPipeline.cu:2018-2023
        const double glare = (double)glare_percent * 0.01;
        xyz[0] += glare * (double)p.scan_illuminant_xyz[0];
        xyz[1] += glare * (double)p.scan_illuminant_xyz[1];
        xyz[2] += glare * (double)p.scan_illuminant_xyz[2];
    }
    double ad[3];
    mat3_apply_d(p.cat02, xyz, ad);
    mat3_apply_d(p.xyz_to_rgb, ad, rgb);
    if (!isfinite(rgb[0]) || !isfinite(rgb[1]) || !isfinite(rgb[2])) return false;
    if (p.gamut_active) {
        float f[3] = {(float)rgb[0], (float)rgb[1], (float)rgb[2]};
        gamut_compress(p, f);
        if (!isfinite(f[0]) || !isfinite(f[1]) || !isfinite(f[2])) return false;
        rgb[0] = f[0];
        rgb[1] = f[1];
        rgb[2] = f[2];
    }
    return true;
}

} // namespace fjb
