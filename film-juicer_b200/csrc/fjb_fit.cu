// fjb_fit.cu -- the per-pixel render chain as a function of fitting parameters, and its
// hand-written adjoint (vector-Jacobian product), for fitting a recipe to target renders.
//
// The chain is the one the render path runs for a pixel (fjb_pixel_math.cuh; reference
// src/Cuda/JuicerCudaDeviceHelpers.cuh:563-1071 and src/Cuda/Scan/JuicerCudaScanPipeline.cu:
// 1700-1811): camera exposure, film curves, runtime DIR (negative donor Langmuir, the
// coupler matrix, the compensated curves), on the print route the 81-wavelength print
// exposure, print curves, then the scanner PCHIP LUT, the scanner correction and the
// CAT02 / output matrices. Its output is the scanner's linear output RGB (before output
// gamut compression and encoding). The parameters theta (FjbFitParams order) enter as
//   exposure_ev[c]    film exposure of layer c (B, G, R) times 2^ev
//   film_gamma[c]     the gamma factor of the film and compensated curves of layer c
//   print_gamma[c]    a gamma factor on the print curve of dye c (C, M, Y), 1 = none
//   donor_k[c]        the donor Langmuir knee of layer c
//   print_ev          print exposure times 2^ev
// The adjoint recomputes each pixel's forward values (the 81 print transmittances
// included) in registers instead of storing them, then runs the chain backwards:
// matrices, correction, exp2, the tricubic Hermite LUT (partials per coordinate), the
// print curves, log10, the spectral sum (d raw / d density = sum_l T S nd ln 2), the
// compensated curves, the coupler matrix and Langmuir terms, the film curves, log10,
// the exposure scale. Piecewise-linear curves contribute their interval slope (zero
// outside the sampled domain); clamped LUT coordinates and values contribute zero.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "../../include/juicer_b200.h"
#include "fjb_internal.h"
#include "fjb_launches.h"
#include "fjb_pixel_math.cuh"
#include "fjb_recipe.h"
#include "fjb_schedule.h"

namespace fjb {

namespace {

constexpr int kFitThreads = 256;
static_assert((kFitThreads & (kFitThreads - 1)) == 0, "the block sum is a power-of-two tree");
// Per-thread gradient sums (a thread adds a few tens of pixels); blocks sum in FP64.
using FitAcc = float;
constexpr float kLn2 = 0.69314718055994530942f;
constexpr float kLn10 = 2.30258509299404568402f;

struct FitTheta {
    float ev[3], gamma[3], pgamma[3], k[3], pev;
};

// Curve value and its slope dy / dxq at xq = logE * gamma (the interval the render
// path's curve_sample selects; slope 0 at and beyond the sampled ends). `knot` and
// `frac` receive the interval's left sample and the position in it (knot -1 outside).
__device__ float curve_with_slope(const float* __restrict__ blob, const CurveRef& c, float logE, float gamma,
                                  float& slope, int& knot, float& frac) {
    slope = 0.0f;
    knot = -1;
    frac = 0.0f;
    if (!isfinite(logE)) return nanf("");
    const float* x = blob + c.x;
    const float* y = blob + c.y;
    const int last = c.n - 1;
    const float xq = logE * gamma;
    if (!(x[last] >= x[0])) return y[0];
    if (xq <= x[0]) return y[0];
    if (xq >= x[last]) return y[last];
    const int i1 = curve_interval_search(x, last, xq);
    if (i1 > last) return y[last];
    const int i0 = i1 - 1;
    const float den = x[i1] - x[i0];
    if (!(den > 0.0f) || !isfinite(den)) return y[i0];
    slope = (y[i1] - y[i0]) / den;
    const float t = (xq - x[i0]) / den;
    knot = i0;
    frac = t;
    return y[i0] + t * (y[i1] - y[i0]);
}

__device__ __forceinline__ double langmuir_d(double v, double k, double r) { return v * (k + r) / (k + v); }

// d Langmuir(v, k, r) / d k
__device__ __forceinline__ float langmuir_dk(float v, float k, float r) {
    const float den = k + v;
    return v * (v - r) / (den * den);
}

__device__ __forceinline__ float hermite_dt(float y0, float y1, float m0, float m1, float t) {
    const float t2 = t * t;
    return (6.0f * t2 - 6.0f * t) * y0 + (3.0f * t2 - 4.0f * t + 1.0f) * m0 + (-6.0f * t2 + 6.0f * t) * y1 +
           (3.0f * t2 - 2.0f * t) * m1;
}

// PCHIP coordinate with its derivative d frac / d normalized (0 when clamped).
__device__ __forceinline__ void coord_d(float nrm, int res, int& base, float& frac, float& dfrac) {
    const float top = (float)(res - 1);
    float coord = nrm * top;
    dfrac = (coord > 0.0f && coord < top) ? top : 0.0f;
    coord = fminf(top, fmaxf(0.0f, coord));
    if (coord >= top) {
        base = res - 2;
        frac = 1.0f;
        return;
    }
    base = (int)floorf(coord);
    frac = coord - (float)base;
}

// scan_lut_sample with the partials of each output (log2 X, Y, Z) with respect to the
// three normalized densities.
__device__ bool scan_lut_sample_d(const PixelParams& p, const double n[3], float out[3], float dout[3][3]) {
    if (!isfinite(n[0]) || !isfinite(n[1]) || !isfinite(n[2]) || p.scan_res < 2) return false;
    const int r = p.scan_res;
    int c, m, y;
    float tc, tm, ty, dc, dm, dy;
    coord_d((float)n[0], r, c, tc, dc);
    coord_d((float)n[1], r, m, tm, dm);
    coord_d((float)n[2], r, y, ty, dy);
    const int s = r - 1;
    const float4* cell = p.scan_cells + 2 * ((c * s + m) * s + y);
    const float4 cmin = __ldg(cell), cmax = __ldg(cell + 1);
    const float lo[3] = {cmin.x, cmin.y, cmin.z};
    const float hi[3] = {cmin.w, cmax.x, cmax.y};
    const int n000 = (c * r + m) * r + y, sc = r * r, sm = r;
    const float hty[4] = {2.0f * ty * ty * ty - 3.0f * ty * ty + 1.0f, ty * ty * ty - 2.0f * ty * ty + ty,
                          -2.0f * ty * ty * ty + 3.0f * ty * ty, ty * ty * ty - ty * ty};
    const float htm[4] = {2.0f * tm * tm * tm - 3.0f * tm * tm + 1.0f, tm * tm * tm - 2.0f * tm * tm + tm,
                          -2.0f * tm * tm * tm + 3.0f * tm * tm, tm * tm * tm - tm * tm};
    for (int o = 0; o < 3; ++o) {
        const float4 a000 = __ldg(p.scan_nodes + 3 * (n000) + o), a100 = __ldg(p.scan_nodes + 3 * (n000 + sc) + o);
        const float4 a010 = __ldg(p.scan_nodes + 3 * (n000 + sm) + o);
        const float4 a110 = __ldg(p.scan_nodes + 3 * (n000 + sc + sm) + o);
        const float4 a001 = __ldg(p.scan_nodes + 3 * (n000 + 1) + o);
        const float4 a101 = __ldg(p.scan_nodes + 3 * (n000 + sc + 1) + o);
        const float4 a011 = __ldg(p.scan_nodes + 3 * (n000 + sm + 1) + o);
        const float4 a111 = __ldg(p.scan_nodes + 3 * (n000 + sc + sm + 1) + o);
        const float v000 = hermite(a000.x, a100.x, a000.y, a100.y, tc), v010 = hermite(a010.x, a110.x, a010.y, a110.y, tc);
        const float v001 = hermite(a001.x, a101.x, a001.y, a101.y, tc), v011 = hermite(a011.x, a111.x, a011.y, a111.y, tc);
        const float d000 = hermite_dt(a000.x, a100.x, a000.y, a100.y, tc), d010 = hermite_dt(a010.x, a110.x, a010.y, a110.y, tc);
        const float d001 = hermite_dt(a001.x, a101.x, a001.y, a101.y, tc), d011 = hermite_dt(a011.x, a111.x, a011.y, a111.y, tc);
        const float sm00 = lerp_ref(a000.z, a100.z, tc), sm10 = lerp_ref(a010.z, a110.z, tc);
        const float sm01 = lerp_ref(a001.z, a101.z, tc), sm11 = lerp_ref(a011.z, a111.z, tc);
        const float vy0 = hermite(v000, v010, sm00, sm10, tm), vy1 = hermite(v001, v011, sm01, sm11, tm);
        const float ay0 = lerp_ref(a000.w, a100.w, tc), by0 = lerp_ref(a010.w, a110.w, tc);
        const float ay1 = lerp_ref(a001.w, a101.w, tc), by1 = lerp_ref(a011.w, a111.w, tc);
        const float sy0 = lerp_ref(ay0, by0, tm), sy1 = lerp_ref(ay1, by1, tm);
        const float v = hermite(vy0, vy1, sy0, sy1, ty);
        out[o] = fminf(hi[o], fmaxf(lo[o], v));
        const bool live = v > lo[o] && v < hi[o];
        // d / d ty
        const float g_ty = hermite_dt(vy0, vy1, sy0, sy1, ty);
        // d / d tm: through vy0, vy1 (Hermite in tm) and sy0, sy1 (lerp in tm)
        const float dvy0_tm = hermite_dt(v000, v010, sm00, sm10, tm), dvy1_tm = hermite_dt(v001, v011, sm01, sm11, tm);
        const float g_tm = hty[0] * dvy0_tm + hty[2] * dvy1_tm + hty[1] * (by0 - ay0) + hty[3] * (by1 - ay1);
        // d / d tc: through every corner Hermite and slope lerp
        const float dvy0_tc = htm[0] * d000 + htm[2] * d010 + htm[1] * (a100.z - a000.z) + htm[3] * (a110.z - a010.z);
        const float dvy1_tc = htm[0] * d001 + htm[2] * d011 + htm[1] * (a101.z - a001.z) + htm[3] * (a111.z - a011.z);
        const float dsy0_tc = (1.0f - tm) * (a100.w - a000.w) + tm * (a110.w - a010.w);
        const float dsy1_tc = (1.0f - tm) * (a101.w - a001.w) + tm * (a111.w - a011.w);
        const float g_tc = hty[0] * dvy0_tc + hty[2] * dvy1_tc + hty[1] * dsy0_tc + hty[3] * dsy1_tc;
        dout[o][0] = live ? g_tc * dc : 0.0f;
        dout[o][1] = live ? g_tm * dm : 0.0f;
        dout[o][2] = live ? g_ty * dy : 0.0f;
    }
    return true;
}

// The print's spectral integral raw_c = sum_l T(l) sens_c(l), T(l) = 2^(D . nd(l)) (the
// film base folded into sens, fjb_params.h),
// evaluated as print_spectral evaluates it (same operations and partial sums), with the
// moments q[3c + j] = sum_l T(l) sens_c(l) nd_j(l) of the same pass: d raw_c / d D_j =
// q[3c + j] ln 2. One exp2 per wavelength serves the value and its derivative.
__device__ __forceinline__ void print_spectral_moments(const PrintSpectral& s, const float d[3], float raw[3],
                                                       float q[9]) {
    float a0[3] = {0.0f, 0.0f, 0.0f}, a1[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 9; ++k) q[k] = 0.0f;
#pragma unroll
    for (int i = 0; i < kSpectralSamples; ++i) {
        const float dl = fmaf(d[0], s.nd[i][0], fmaf(d[1], s.nd[i][1], d[2] * s.nd[i][2]));
        const float t = mufu_exp2(dl);
        float* a = (i & 1) ? a1 : a0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a[c] = fmaf(t, s.sens[i][c], a[c]);
            const float w = t * s.sens[i][c];
            q[3 * c + 0] = fmaf(w, s.nd[i][0], q[3 * c + 0]);
            q[3 * c + 1] = fmaf(w, s.nd[i][1], q[3 * c + 1]);
            q[3 * c + 2] = fmaf(w, s.nd[i][2], q[3 * c + 2]);
        }
    }
    raw[0] = a0[0] + a1[0];
    raw[1] = a0[1] + a1[1];
    raw[2] = a0[2] + a1[2];
}

// One pixel: the linear output RGB for theta; with kGrad, also adds the pixel's
// vector-Jacobian product g_rgb^T d rgb / d theta into g_th (FjbFitParams order).
// False for a pixel the chain rejects (non-finite values, LUT failure); a rejected
// pixel adds nothing (every rejection comes before the adjoint part).
// `e0`: the pixel's film exposure B, G, R before the exposure parameters. `dldk` (kGrad
// with negative-donor DIR): d L(y_d[i], k_d) / d k_d for every donor d and knot i of the
// compensated curves, [d * n + i]. `g_e0` (kGrad, may be null) receives the gradient
// with respect to e0.
// kSpatial (spatial DIR): the DIR corrections of the B, G, R receivers are the filtered
// planes' values `cf` instead of the pixel's own donors (the capture development of
// src/Cuda/JuicerCudaDeviceHelpers.cuh:1267-1328); the adjoint writes d / d cf into
// `g_cf` and leaves the donors to the source stage's adjoint.
template <bool kPrint, bool kGrad, bool kSpatial = false>
__device__ bool fit_pixel(const PixelParams& p, const float* __restrict__ blob, const FitTheta& th, const float e0[3],
                          double rgb[3], const float* g_rgb, FitAcc* g_th, const float* __restrict__ dldk,
                          float* g_e0, const float* cf = nullptr, float* g_cf = nullptr) {
    // ---- forward, keeping what the adjoint needs ----
    float e[3], logS[3], layer[3], sl[3];
    for (int c = 0; c < 3; ++c) {
        e[c] = e0[c] * exp2f(th.ev[c]);
        logS[c] = log_exposure(e[c]);
        if (!isfinite(logS[c])) return false;
        int kn;
        float fr;
        layer[c] = curve_with_slope(blob, p.film_curve[c], logS[c], th.gamma[c], sl[c], kn, fr);
    }
    float D[3], logC[3] = {0.0f, 0.0f, 0.0f}, sd[3] = {0.0f, 0.0f, 0.0f}, dv[3] = {0.0f, 0.0f, 0.0f},
                dk[3] = {0.0f, 0.0f, 0.0f}, dfr[3] = {0.0f, 0.0f, 0.0f};
    int dkn[3] = {-1, -1, -1};
    const bool dir = p.dir_mode == kDirNegativeDonor || p.dir_mode == kDirPositiveReceiver;
    const bool positive = p.dir_mode == kDirPositiveReceiver;
    // positive stocks: d (finalised correction) / d (coupler sum) per receiver
    float dfin[3] = {1.0f, 1.0f, 1.0f};
    if (dir) {
        float corr[3];
        if constexpr (kSpatial) {
            for (int j = 0; j < 3; ++j) {
                corr[j] = cf[j];
                if (!isfinite(corr[j])) return false;
            }
        } else {
            float donor[3];
            for (int c = 0; c < 3; ++c) {
                const float v = layer[c];
                if (positive) {
                    // the donor is the density still to form (src/Cuda/JuicerCudaDeviceHelpers.cuh:1173)
                    donor[c] = p.dir_dmax[c] - v;
                    dv[c] = -1.0f;
                    dk[c] = 0.0f;
                } else {
                    const float k = th.k[c], r = p.dir_dref[c];
                    const float den = k + v;
                    donor[c] = v * (k + r) / den;
                    dv[c] = k * (k + r) / (den * den);
                    dk[c] = v * (v - r) / (den * den);
                }
                if (!isfinite(donor[c])) return false;
            }
            const float* M = p.dir_m;
            for (int j = 0; j < 3; ++j) corr[j] = M[j] * donor[0] + M[3 + j] * donor[1] + M[6 + j] * donor[2];
        }
        if (positive) {
            // receiver Langmuir: c (kr + cref) / (kr + c), zero where the receiver has no reference
            for (int j = 0; j < 3; ++j) {
                const float cref = p.dir_receiver_cref[j], kr = p.dir_receiver_kr[j];
                if (cref == 0.0f) {
                    corr[j] = 0.0f;
                    dfin[j] = 0.0f;
                    continue;
                }
                const float c = corr[j], den = kr + c;
                corr[j] = c * (kr + cref) / den;
                dfin[j] = kr * (kr + cref) / (den * den);
                if (!isfinite(corr[j]) || !isfinite(dfin[j])) return false;
            }
        }
        for (int j = 0; j < 3; ++j) {
            logC[j] = logS[j] - corr[j];
            D[2 - j] = curve_with_slope(blob, p.dir_curve[j], logC[j], th.gamma[j], sd[j], dkn[j], dfr[j]);
        }
    } else {
        for (int c = 0; c < 3; ++c) D[2 - c] = layer[c];
    }
    float scanD[3], rawp[3] = {0.0f, 0.0f, 0.0f}, lp[3] = {0.0f, 0.0f, 0.0f}, sp[3] = {0.0f, 0.0f, 0.0f};
    float q[9];
    float raw_scale = 0.0f;
    if constexpr (kPrint) {
        if (!(isfinite(D[0]) && isfinite(D[1]) && isfinite(D[2]))) return false;
        float raw[3];
        if constexpr (kGrad) {
            print_spectral_moments(p.spectral, D, raw, q);
        } else {
            print_spectral(p.spectral, D, raw);
        }
        const float spev = exp2f(th.pev);
        raw_scale = p.print_midgray * p.print_exposure * spev * p.print_route_correction;
        const float pf = p.print_preflash_exposure;
        for (int c = 0; c < 3; ++c) {
            float v = raw[c] * p.print_midgray;
            if (isfinite(pf) && pf > 0.0f) v += p.print_preflash_raw[c] * pf;
            v *= p.print_exposure;
            v *= spev;
            v *= p.print_route_correction;
            rawp[c] = v;
            lp[c] = log10f(v + 1e-10f);
            int kn;
            float fr;
            scanD[c] = curve_with_slope(blob, p.print_curve[c], lp[c], th.pgamma[c], sp[c], kn, fr);
        }
    } else {
        for (int c = 0; c < 3; ++c) scanD[c] = D[c];
    }
    double nd[3];
    for (int c = 0; c < 3; ++c)
        nd[c] = p.scan_medium_negative ? ((double)scanD[c] + (double)p.scan_min_cmy[c]) * (double)p.scan_inv_span_cmy[c]
                                       : ((double)scanD[c] - (double)p.scan_min_cmy[c]) * (double)p.scan_inv_span_cmy[c];
    float l2[3], dl2[3][3];
    if constexpr (kGrad) {
        if (!scan_lut_sample_d(p, nd, l2, dl2)) return false;
    } else {
        if (!scan_lut_sample(p, nd, l2)) return false;
    }
    double xyz[3] = {(double)exp2f(l2[0]), (double)exp2f(l2[1]), (double)exp2f(l2[2])};
    double xc[3] = {xyz[0], xyz[1], xyz[2]}, sc = 1.0, dsc = 0.0;
    if (p.correction_active) {
        const double t = (double)p.correction_slope * xyz[1] + (double)p.correction_offset;
        const double cy = fmin(fmax(t, 0.0), 1.0);
        const double den = xyz[1] + 1e-10;
        sc = cy / den;
        const double dcy = (t > 0.0 && t < 1.0) ? (double)p.correction_slope : 0.0;
        dsc = (dcy * den - cy) / (den * den);
        for (int c = 0; c < 3; ++c) xc[c] = xyz[c] * sc;
    }
    double ad[3];
    mat3_apply_d(p.cat02, xc, ad);
    mat3_apply_d(p.xyz_to_rgb, ad, rgb);
    if (!isfinite(rgb[0]) || !isfinite(rgb[1]) || !isfinite(rgb[2])) return false;
    if constexpr (!kGrad) return true;

    // ---- adjoint (FP32 per pixel; the caller sums pixels in FP64) ----
    float g_ad[3], g_xc[3], g_xyz[3];
    for (int c = 0; c < 3; ++c) g_ad[c] = p.xyz_to_rgb[c] * g_rgb[0] + p.xyz_to_rgb[3 + c] * g_rgb[1] +
                                          p.xyz_to_rgb[6 + c] * g_rgb[2];
    for (int c = 0; c < 3; ++c) g_xc[c] = p.cat02[c] * g_ad[0] + p.cat02[3 + c] * g_ad[1] + p.cat02[6 + c] * g_ad[2];
    if (p.correction_active) {
        const float dot = (float)(g_xc[0] * xyz[0] + g_xc[1] * xyz[1] + g_xc[2] * xyz[2]);
        for (int c = 0; c < 3; ++c) g_xyz[c] = g_xc[c] * (float)sc;
        g_xyz[1] += dot * (float)dsc;
    } else {
        for (int c = 0; c < 3; ++c) g_xyz[c] = g_xc[c];
    }
    float g_l2[3];
    for (int o = 0; o < 3; ++o) g_l2[o] = g_xyz[o] * (float)xyz[o] * kLn2;
    float g_scan[3];
    for (int c = 0; c < 3; ++c)
        g_scan[c] = (g_l2[0] * dl2[0][c] + g_l2[1] * dl2[1][c] + g_l2[2] * dl2[2][c]) * p.scan_inv_span_cmy[c];
    float g_D[3];
    if constexpr (kPrint) {
        float g_raw[3], g_pev = 0.0f;
        for (int c = 0; c < 3; ++c) {
            const float g_lp = g_scan[c] * sp[c] * th.pgamma[c];
            g_th[6 + c] += (g_scan[c] * sp[c] * lp[c]);
            const float g_rawp = g_lp / ((rawp[c] + 1e-10f) * kLn10);
            g_pev += g_rawp * rawp[c] * kLn2;
            g_raw[c] = g_rawp * raw_scale;
        }
        g_th[12] += g_pev;
        for (int j = 0; j < 3; ++j) g_D[j] = (g_raw[0] * q[j] + g_raw[1] * q[3 + j] + g_raw[2] * q[6 + j]) * kLn2;
    } else {
        for (int c = 0; c < 3; ++c) g_D[c] = g_scan[c];
    }
    float g_logS[3], g_layer[3];
    if (dir) {
        float g_corr[3];
        for (int j = 0; j < 3; ++j) {
            const float g = g_D[2 - j];
            const float g_logC = g * sd[j] * th.gamma[j];
            g_th[3 + j] += (g * sd[j] * logC[j]);
            g_logS[j] = g_logC;
            g_corr[j] = -g_logC * dfin[j];
        }
        const float* M = p.dir_m;
        if constexpr (kSpatial) {
            for (int j = 0; j < 3; ++j) {
                g_cf[j] = g_corr[j];
                g_layer[j] = 0.0f;
            }
        } else {
            for (int i = 0; i < 3; ++i) {
                const float g_donor = M[3 * i] * g_corr[0] + M[3 * i + 1] * g_corr[1] + M[3 * i + 2] * g_corr[2];
                g_layer[i] = g_donor * dv[i];
                g_th[9 + i] += (g_donor * dk[i]);
            }
        }
        // The compensated axes depend on the knees (axis_j[i] = logE[i] - sum_d M[d][j]
        // L(y_d[i], k_d)): d D / d axis at the interval's knots is -slope (1 - t), -slope t.
        // (Positive stocks have no donor knees: their axes are the recipe's.)
        const int n = p.dir_curve[0].n;
        for (int j = 0; j < 3; ++j) {
            if (positive || dkn[j] < 0) continue;
            const float w = g_D[2 - j] * sd[j];
            const int i0 = dkn[j];
            const float t = dfr[j];
            for (int d = 0; d < 3; ++d) {
                const float s0 = dldk[d * n + i0], s1 = dldk[d * n + i0 + 1];
                g_th[9 + d] += (w * M[3 * d + j] * ((1.0f - t) * s0 + t * s1));
            }
        }
    } else {
        for (int c = 0; c < 3; ++c) {
            g_layer[c] = g_D[2 - c];
            g_logS[c] = 0.0f;
        }
    }
    for (int c = 0; c < 3; ++c) {
        g_logS[c] += g_layer[c] * sl[c] * th.gamma[c];
        g_th[3 + c] += (g_layer[c] * sl[c] * logS[c]);
        const float g_e = e[c] > 0.0f ? g_logS[c] / ((e[c] + 1e-10f) * kLn10) : 0.0f;
        g_th[c] += (g_e * e[c] * kLn2);
        if (g_e0) g_e0[c] = g_e * exp2f(th.ev[c]);
    }
    return true;
}

// Stages the curve blob into shared memory (as the pixel-chain kernels do). With donor
// knees other than the recipe's, the DIR compensated axes are moved by the change of
// the Langmuir donors at each sample, in FP64:
//   axis_j[i] += sum_d M[d][j] (L(y_d[i], k0_d) - L(y_d[i], k_d))
// (the host builds axis_j[i] = logE[i] - sum_d M[d][j] L(y_d[i], k0_d):
// rust/film-juicer-core/src/film/dir.rs:258-290). The recipe's knees leave them as given.
__device__ __forceinline__ const float* stage_blob(const PixelParams& p, const FitTheta& th, float* smem) {
    const float4* g = reinterpret_cast<const float4*>(p.curve_blob);
    float4* s4 = reinterpret_cast<float4*>(smem);
    for (int i = threadIdx.x; i < (p.curve_blob_floats >> 2); i += blockDim.x) s4[i] = __ldg(g + i);
    __syncthreads();
    if (p.dir_mode == kDirNegativeDonor &&
        (th.k[0] != p.dir_donor_k[0] || th.k[1] != p.dir_donor_k[1] || th.k[2] != p.dir_donor_k[2])) {
        const int n = p.dir_curve[0].n;
        for (int e = threadIdx.x; e < 3 * n; e += blockDim.x) {
            const int j = e / n, i = e - j * n;
            double delta = 0.0;
            for (int d = 0; d < 3; ++d) {
                const double y = (double)smem[p.film_curve[d].y + i], r = (double)p.dir_dref[d];
                delta += (double)p.dir_m[3 * d + j] *
                         (langmuir_d(y, (double)p.dir_donor_k[d], r) - langmuir_d(y, (double)th.k[d], r));
            }
            float* ax = smem + p.dir_curve[j].x;
            ax[i] = (float)((double)ax[i] + delta);
        }
        __syncthreads();
    }
    return smem;
}

// Floats of the staged curve blob (a whole number of float4s).
__host__ __device__ __forceinline__ int fit_blob_floats(const PixelParams& p) { return (p.curve_blob_floats >> 2) << 2; }

// Dynamic shared memory of the adjoint: the curve blob, then the knee-derivative table.
inline size_t fit_vjp_smem(const PixelParams& p) {
    const int n = p.dir_mode == kDirNegativeDonor ? p.dir_curve[0].n : 0;
    return ((size_t)fit_blob_floats(p) + 3 * (size_t)n) * sizeof(float);
}

// Carrier-plane input (film exposure B, G, R before the route correction, as the
// camera exposure stage writes it) and, for the adjoint, the optional gradient planes
// with respect to it.
struct FitCarrier {
    const float* b;
    const float* g;
    const float* r;
    long long stride;
    float* gb;
    float* gg;
    float* gr;
    // spatial DIR: the filtered corrections of the B, G, R receivers (the Y, M, C
    // planes of the spatial-DIR stage) and, for the adjoint, their gradient planes;
    // all with the carrier's stride
    const float* fy = nullptr;
    const float* fm = nullptr;
    const float* fc = nullptr;
    float* gfy = nullptr;
    float* gfm = nullptr;
    float* gfc = nullptr;
};

// The film exposure e0 (B, G, R) of pixel idx: from the source RGB through the camera
// exposure, or from the carrier planes as the capture stage reads them
// (max(0, carrier x route correction)).
template <bool kCarrier>
__device__ __forceinline__ void load_exposure(const PixelParams& p, const FitCarrier& cr, long long idx, float e0[3]) {
    const int y = (int)(idx / p.width), x = (int)(idx - (long long)y * p.width);
    if constexpr (kCarrier) {
        const long long ci = (long long)y * cr.stride + x;
        e0[0] = fmaxf(0.0f, cr.b[ci] * p.route_correction_scale);
        e0[1] = fmaxf(0.0f, cr.g[ci] * p.route_correction_scale);
        e0[2] = fmaxf(0.0f, cr.r[ci] * p.route_correction_scale);
    } else {
        const float* s =
            reinterpret_cast<const float*>(p.src + (long long)y * p.src_row_bytes) + (long long)x * p.components;
        const float in[3] = {s[0], s[1], s[2]};
        camera_linear_exposure(p, in, true, e0);
    }
}

// The filtered DIR corrections of pixel idx (spatial DIR, carrier layout).
__device__ __forceinline__ void load_filtered(const PixelParams& p, const FitCarrier& cr, long long idx, float cf[3]) {
    const int y = (int)(idx / p.width), x = (int)(idx - (long long)y * p.width);
    const long long ci = (long long)y * cr.stride + x;
    cf[0] = cr.fy[ci];
    cf[1] = cr.fm[ci];
    cf[2] = cr.fc[ci];
}

// Linear output RGB planes for theta (NaN where the chain rejects a pixel).
template <bool kPrint, bool kCarrier, bool kSpatial = false>
__global__ void __launch_bounds__(kFitThreads, 2) fit_forward_kernel(const __grid_constant__ PixelParams p, FitTheta th,
                                                                  FitCarrier cr, float* out_r, float* out_g,
                                                                  float* out_b) {
    extern __shared__ float4 fit_smem4[];
    const float* blob = stage_blob(p, th, reinterpret_cast<float*>(fit_smem4));
    const long long total = (long long)p.width * p.height;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        float e0[3], cf[3] = {0.0f, 0.0f, 0.0f};
        load_exposure<kCarrier>(p, cr, idx, e0);
        if constexpr (kSpatial) load_filtered(p, cr, idx, cf);
        double rgb[3];
        const bool ok =
            fit_pixel<kPrint, false, kSpatial>(p, blob, th, e0, rgb, nullptr, nullptr, nullptr, nullptr, cf, nullptr);
        out_r[idx] = ok ? (float)rgb[0] : nanf("");
        out_g[idx] = ok ? (float)rgb[1] : nanf("");
        out_b[idx] = ok ? (float)rgb[2] : nanf("");
    }
}

constexpr int kFitParams = 13;

// Per-block sums (FP64, fixed order) of the pixels' vector-Jacobian products; with
// carrier input and gradient planes, also d <g, rgb> / d carrier per pixel (zero where
// the chain rejects the pixel or the cotangent is zero).
template <bool kPrint, bool kCarrier, bool kSpatial = false>
__global__ void __launch_bounds__(kFitThreads, 2) fit_vjp_kernel(const __grid_constant__ PixelParams p, FitTheta th,
                                                              FitCarrier cr, const float* __restrict__ g_r,
                                                              const float* __restrict__ g_g,
                                                              const float* __restrict__ g_b, double* partials) {
    extern __shared__ float4 fit_smem4[];
    const float* blob = stage_blob(p, th, reinterpret_cast<float*>(fit_smem4));
    float* dldk = reinterpret_cast<float*>(fit_smem4) + fit_blob_floats(p);
    if (p.dir_mode == kDirNegativeDonor) {
        const int n = p.dir_curve[0].n;
        for (int e = threadIdx.x; e < 3 * n; e += blockDim.x) {
            const int d = e / n, i = e - d * n;
            dldk[e] = langmuir_dk(blob[p.film_curve[d].y + i], th.k[d], p.dir_dref[d]);
        }
        __syncthreads();
    }
    __shared__ double red[kFitThreads];
    FitAcc acc[kFitParams];
    for (int k = 0; k < kFitParams; ++k) acc[k] = 0.0f;
    const bool carrier_grad = kCarrier && cr.gb != nullptr;
    const long long total = (long long)p.width * p.height;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const float g[3] = {g_r[idx], g_g[idx], g_b[idx]};
        float ge[3] = {0.0f, 0.0f, 0.0f}, gcf[3] = {0.0f, 0.0f, 0.0f};
        float e0[3] = {0.0f, 0.0f, 0.0f};
        if (g[0] != 0.0f || g[1] != 0.0f || g[2] != 0.0f) {
            load_exposure<kCarrier>(p, cr, idx, e0);
            float cf[3] = {0.0f, 0.0f, 0.0f};
            if constexpr (kSpatial) load_filtered(p, cr, idx, cf);
            double rgb[3];
            if (!fit_pixel<kPrint, true, kSpatial>(p, blob, th, e0, rgb, g, acc, dldk, carrier_grad ? ge : nullptr, cf,
                                                   gcf)) {
                ge[0] = ge[1] = ge[2] = 0.0f;
                gcf[0] = gcf[1] = gcf[2] = 0.0f;
            }
        }
        if constexpr (kSpatial) {
            const int y = (int)(idx / p.width), x = (int)(idx - (long long)y * p.width);
            const long long ci = (long long)y * cr.stride + x;
            cr.gfy[ci] = gcf[0];
            cr.gfm[ci] = gcf[1];
            cr.gfc[ci] = gcf[2];
        }
        if (carrier_grad) {
            // e0 = max(0, carrier x route): the route factor inside, zero where clamped
            const int y = (int)(idx / p.width), x = (int)(idx - (long long)y * p.width);
            const long long ci = (long long)y * cr.stride + x;
            const float rc = p.route_correction_scale;
            cr.gb[ci] = e0[0] > 0.0f ? ge[0] * rc : 0.0f;
            cr.gg[ci] = e0[1] > 0.0f ? ge[1] * rc : 0.0f;
            cr.gr[ci] = e0[2] > 0.0f ? ge[2] * rc : 0.0f;
        }
    }
    for (int k = 0; k < kFitParams; ++k) {
        red[threadIdx.x] = (double)acc[k];
        __syncthreads();
        for (int s = kFitThreads / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * kFitParams + k] = red[0];
        __syncthreads();
    }
}

__global__ void fit_reduce_kernel(const double* __restrict__ partials, int blocks, double* out) {
    const int k = threadIdx.x;
    if (k >= kFitParams) return;
    double s = 0.0;
    for (int b = 0; b < blocks; ++b) s += partials[(size_t)b * kFitParams + k];
    out[k] = s;
}

// Spatial-DIR source of one pixel for theta (src/Cuda/Film/JuicerCudaFilmPipeline.cu:124-214):
// the film exposure, the pre-DIR layer densities and the donor corrections they
// release to the B, G, R receivers, corr_j = sum_d M[d][j] donor_d (donor_d = L(layer_d, k_d),
// or dmax_d - layer_d for positive stocks; the receiver Langmuir follows the filter). With kGrad,
// adds g_src^T d corr / d theta into g_th and writes d <g_src, corr> / d e0 into g_e0
// (may be null). False (nothing added) where a value is not finite.
template <bool kGrad>
__device__ bool dir_source_pixel(const PixelParams& p, const float* __restrict__ blob, const FitTheta& th,
                                 const float e0[3], float corr[3], const float* g_src, FitAcc* g_th, float* g_e0) {
    float e[3], logS[3], layer[3], sl[3], donor[3], dv[3], dk[3];
    for (int c = 0; c < 3; ++c) {
        e[c] = e0[c] * exp2f(th.ev[c]);
        logS[c] = log_exposure(e[c]);
        if (!isfinite(logS[c])) return false;
        int kn;
        float fr;
        layer[c] = curve_with_slope(blob, p.film_curve[c], logS[c], th.gamma[c], sl[c], kn, fr);
        const float v = layer[c];
        if (p.dir_mode == kDirPositiveReceiver) {
            donor[c] = p.dir_dmax[c] - v;
            dv[c] = -1.0f;
            dk[c] = 0.0f;
        } else {
            const float k = th.k[c], r = p.dir_dref[c];
            const float den = k + v;
            donor[c] = v * (k + r) / den;
            dv[c] = k * (k + r) / (den * den);
            dk[c] = v * (v - r) / (den * den);
        }
        if (!isfinite(donor[c])) return false;
    }
    const float* M = p.dir_m;
    for (int j = 0; j < 3; ++j) {
        corr[j] = M[j] * donor[0] + M[3 + j] * donor[1] + M[6 + j] * donor[2];
        if (!isfinite(corr[j])) return false;
    }
    if constexpr (kGrad) {
        for (int i = 0; i < 3; ++i) {
            const float g_donor = M[3 * i] * g_src[0] + M[3 * i + 1] * g_src[1] + M[3 * i + 2] * g_src[2];
            const float g_layer = g_donor * dv[i];
            g_th[9 + i] += (g_donor * dk[i]);
            const float g_logS = g_layer * sl[i] * th.gamma[i];
            g_th[3 + i] += (g_layer * sl[i] * logS[i]);
            const float g_e = e[i] > 0.0f ? g_logS / ((e[i] + 1e-10f) * kLn10) : 0.0f;
            g_th[i] += (g_e * e[i] * kLn2);
            if (g_e0) g_e0[i] = g_e * exp2f(th.ev[i]);
        }
    }
    return true;
}

// The source stage's correction planes (B, G, R receivers into cr.gfy/gfm/gfc's
// layout: the Y, M, C planes), NaN where a pixel's source is not finite.
template <bool kCarrier>
__global__ void __launch_bounds__(kFitThreads, 2) fit_dir_source_kernel(const __grid_constant__ PixelParams p,
                                                                     FitTheta th, FitCarrier cr, float* out_y,
                                                                     float* out_m, float* out_c) {
    extern __shared__ float4 fit_smem4[];
    const float* blob = stage_blob(p, th, reinterpret_cast<float*>(fit_smem4));
    const long long total = (long long)p.width * p.height;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        float e0[3], corr[3];
        load_exposure<kCarrier>(p, cr, idx, e0);
        const bool ok = dir_source_pixel<false>(p, blob, th, e0, corr, nullptr, nullptr, nullptr);
        const int y = (int)(idx / p.width), x = (int)(idx - (long long)y * p.width);
        const long long ci = (long long)y * cr.stride + x;
        out_y[ci] = ok ? corr[0] : nanf("");
        out_m[ci] = ok ? corr[1] : nanf("");
        out_c[ci] = ok ? corr[2] : nanf("");
    }
}

// Adjoint of the source stage: per-block FP64 sums of g_src^T d corr / d theta (g_src:
// the cotangents of the correction planes before the spatial filter); with carrier
// gradient planes, adds d <g_src, corr> / d carrier to them.
template <bool kCarrier>
__global__ void __launch_bounds__(kFitThreads, 2) fit_dir_source_vjp_kernel(const __grid_constant__ PixelParams p,
                                                                         FitTheta th, FitCarrier cr,
                                                                         const float* __restrict__ g_y,
                                                                         const float* __restrict__ g_m,
                                                                         const float* __restrict__ g_c,
                                                                         double* partials) {
    extern __shared__ float4 fit_smem4[];
    const float* blob = stage_blob(p, th, reinterpret_cast<float*>(fit_smem4));
    __shared__ double red[kFitThreads];
    FitAcc acc[kFitParams];
    for (int k = 0; k < kFitParams; ++k) acc[k] = 0.0f;
    const bool carrier_grad = kCarrier && cr.gb != nullptr;
    const long long total = (long long)p.width * p.height;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(idx / p.width), x = (int)(idx - (long long)y * p.width);
        const long long ci = (long long)y * cr.stride + x;
        const float g[3] = {g_y[ci], g_m[ci], g_c[ci]};
        if (g[0] == 0.0f && g[1] == 0.0f && g[2] == 0.0f) continue;
        float e0[3], corr[3], ge[3] = {0.0f, 0.0f, 0.0f};
        load_exposure<kCarrier>(p, cr, idx, e0);
        if (!dir_source_pixel<true>(p, blob, th, e0, corr, g, acc, carrier_grad ? ge : nullptr)) continue;
        if (carrier_grad) {
            const float rc = p.route_correction_scale;
            if (e0[0] > 0.0f) cr.gb[ci] += ge[0] * rc;
            if (e0[1] > 0.0f) cr.gg[ci] += ge[1] * rc;
            if (e0[2] > 0.0f) cr.gr[ci] += ge[2] * rc;
        }
    }
    for (int k = 0; k < kFitParams; ++k) {
        red[threadIdx.x] = (double)acc[k];
        __syncthreads();
        for (int s = kFitThreads / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * kFitParams + k] = red[0];
        __syncthreads();
    }
}

int fit_blocks() {
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return (sms > 0 ? sms : 148) * 4;
}

bool theta_from(const FjbFitParams& f, FitTheta& th) {
    for (int c = 0; c < 3; ++c) {
        th.ev[c] = f.exposure_ev[c];
        th.gamma[c] = f.film_gamma[c];
        th.pgamma[c] = f.print_gamma[c];
        th.k[c] = f.donor_k[c];
        if (!std::isfinite(th.ev[c]) || !std::isfinite(th.gamma[c]) || !std::isfinite(th.pgamma[c]) ||
            !(th.k[c] > 0.0f) || !std::isfinite(th.k[c]))
            return false;
    }
    th.pev = f.print_ev;
    return std::isfinite(th.pev);
}

} // namespace

} // namespace fjb

namespace fjb {
namespace {

template <bool kCarrier, bool kSpatial = false>
cudaError_t launch_fit_forward(const PixelParams& p, const FitTheta& th, const FitCarrier& cr, float* out_r,
                               float* out_g, float* out_b, cudaStream_t s) {
    const size_t smem = (size_t)p.curve_blob_floats * sizeof(float);
    count_launch();
    if (p.route == kRoutePrint) {
        auto* k = fit_forward_kernel<true, kCarrier, kSpatial>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<fit_blocks(), kFitThreads, smem, s>>>(p, th, cr, out_r, out_g, out_b);
    } else {
        auto* k = fit_forward_kernel<false, kCarrier, kSpatial>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<fit_blocks(), kFitThreads, smem, s>>>(p, th, cr, out_r, out_g, out_b);
    }
    return cudaGetLastError();
}

template <bool kCarrier, bool kSpatial = false>
cudaError_t launch_fit_vjp(const PixelParams& p, const FitTheta& th, const FitCarrier& cr, const float* grad_r,
                           const float* grad_g, const float* grad_b, double* partials, double* grad_params,
                           cudaStream_t s) {
    const int blocks = fit_blocks();
    const size_t smem = fit_vjp_smem(p);
    count_launch();
    if (p.route == kRoutePrint) {
        auto* k = fit_vjp_kernel<true, kCarrier, kSpatial>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<blocks, kFitThreads, smem, s>>>(p, th, cr, grad_r, grad_g, grad_b, partials);
    } else {
        auto* k = fit_vjp_kernel<false, kCarrier, kSpatial>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<blocks, kFitThreads, smem, s>>>(p, th, cr, grad_r, grad_g, grad_b, partials);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        count_launch();
        fit_reduce_kernel<<<1, 32, 0, s>>>(partials, blocks, grad_params);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_fit_dir_source(const PixelParams& p, const FitTheta& th, const FitCarrier& cr, float* out_y,
                                  float* out_m, float* out_c, cudaStream_t s) {
    const size_t smem = (size_t)p.curve_blob_floats * sizeof(float);
    count_launch();
    auto* k = fit_dir_source_kernel<true>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<fit_blocks(), kFitThreads, smem, s>>>(p, th, cr, out_y, out_m, out_c);
    return cudaGetLastError();
}

cudaError_t launch_fit_dir_source_vjp(const PixelParams& p, const FitTheta& th, const FitCarrier& cr, const float* g_y,
                                      const float* g_m, const float* g_c, double* partials, double* grad_params,
                                      cudaStream_t s) {
    const int blocks = fit_blocks();
    const size_t smem = (size_t)p.curve_blob_floats * sizeof(float);
    count_launch();
    auto* k = fit_dir_source_vjp_kernel<true>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<blocks, kFitThreads, smem, s>>>(p, th, cr, g_y, g_m, g_c, partials);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        count_launch();
        fit_reduce_kernel<<<1, 32, 0, s>>>(partials, blocks, grad_params);
        e = cudaGetLastError();
    }
    return e;
}

} // namespace
} // namespace fjb

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

extern "C" {

size_t fjb_fit_scratch_bytes(void) { return (size_t)fjb::fit_blocks() * fjb::kFitParams * sizeof(double); }

FjStatus fjb_fit_defaults(FjbRecipe* recipe, FjbFitParams* out, FjErrorBuffer* error) {
    if (!recipe || !out) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    const fjb::PixelParams& p = recipe->r.params;
    for (int c = 0; c < 3; ++c) {
        out->exposure_ev[c] = 0.0f;
        out->film_gamma[c] = p.gamma_bgr[c];
        out->print_gamma[c] = 1.0f;
        out->donor_k[c] = p.dir_mode == fjb::kDirNegativeDonor ? p.dir_donor_k[c] : 1.0f;
    }
    out->print_ev = 0.0f;
    write_error(error, "");
    return ok_status();
}

static FjStatus fit_check(FjbRecipe* recipe, const FjbFitParams* params, bool have_input, uint32_t components,
                          int32_t width, int32_t height, fjb::FitTheta& th, FjErrorBuffer* error) {
    if (!recipe || !params || !have_input) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if ((components != 3 && components != 4) || width < 0 || height < 0)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unsupported image geometry");
    const fjb::PixelParams& p = recipe->r.params;
    if (!fjb::theta_from(*params, th))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "fit parameters must be finite, knees positive");
    return ok_status();
}


FjStatus fjb_fit_forward(FjbRecipe* recipe, const FjbFitParams* params, const float* src, ptrdiff_t src_row_bytes,
                         uint32_t components, float* out_r, float* out_g, float* out_b, int32_t width, int32_t height,
                         void* stream, FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = fit_check(recipe, params, src != nullptr, components, width, height, th, error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!out_r || !out_g || !out_b) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if ((long long)width * height > 0) {
        fjb::PixelParams p = recipe->r.params;
        p.src = reinterpret_cast<const char*>(src);
        p.src_row_bytes = src_row_bytes;
        p.components = (int)components;
        p.width = width;
        p.height = height;
        const cudaError_t e = fjb::launch_fit_forward<false>(p, th, fjb::FitCarrier{}, out_r, out_g, out_b,
                                                             reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_status(e, error, "fit forward");
    }
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_fit_vjp(FjbRecipe* recipe, const FjbFitParams* params, const float* src, ptrdiff_t src_row_bytes,
                     uint32_t components, const float* grad_r, const float* grad_g, const float* grad_b,
                     int32_t width, int32_t height, double* grad_params, void* scratch, size_t scratch_bytes,
                     void* stream, FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = fit_check(recipe, params, src != nullptr, components, width, height, th, error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!grad_r || !grad_g || !grad_b || !grad_params || !scratch)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (scratch_bytes < (size_t)fjb::fit_blocks() * fjb::kFitParams * sizeof(double))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "fit scratch smaller than fjb_fit_scratch_bytes()");
    fjb::PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src);
    p.src_row_bytes = src_row_bytes;
    p.components = (int)components;
    p.width = width;
    p.height = height;
    const cudaError_t e =
        fjb::launch_fit_vjp<false>(p, th, fjb::FitCarrier{}, grad_r, grad_g, grad_b, static_cast<double*>(scratch),
                                   grad_params, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "fit adjoint");
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_fit_forward_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                 const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                 float* out_r, float* out_g, float* out_b, int32_t width, int32_t height, void* stream,
                                 FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = fit_check(recipe, params, carrier_b && carrier_g && carrier_r, 3, width, height, th, error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!out_r || !out_g || !out_b || carrier_stride < width)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument or carrier stride below the width");
    if ((long long)width * height > 0) {
        fjb::PixelParams p = recipe->r.params;
        p.width = width;
        p.height = height;
        const fjb::FitCarrier cr{carrier_b, carrier_g, carrier_r, (long long)carrier_stride, nullptr, nullptr, nullptr};
        const cudaError_t e =
            fjb::launch_fit_forward<true>(p, th, cr, out_r, out_g, out_b, reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_status(e, error, "fit forward");
    }
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_fit_vjp_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                             const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                             const float* grad_r, const float* grad_g, const float* grad_b, int32_t width,
                             int32_t height, double* grad_params, float* grad_carrier_b, float* grad_carrier_g,
                             float* grad_carrier_r, void* scratch, size_t scratch_bytes, void* stream,
                             FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = fit_check(recipe, params, carrier_b && carrier_g && carrier_r, 3, width, height, th, error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!grad_r || !grad_g || !grad_b || !grad_params || !scratch || carrier_stride < width)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument or carrier stride below the width");
    const bool planes = grad_carrier_b || grad_carrier_g || grad_carrier_r;
    if (planes && !(grad_carrier_b && grad_carrier_g && grad_carrier_r))
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "carrier gradient planes: all three or none");
    if (scratch_bytes < (size_t)fjb::fit_blocks() * fjb::kFitParams * sizeof(double))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "fit scratch smaller than fjb_fit_scratch_bytes()");
    fjb::PixelParams p = recipe->r.params;
    p.width = width;
    p.height = height;
    const fjb::FitCarrier cr{carrier_b,      carrier_g,      carrier_r,     (long long)carrier_stride,
                             grad_carrier_b, grad_carrier_g, grad_carrier_r};
    const cudaError_t e =
        fjb::launch_fit_vjp<true>(p, th, cr, grad_r, grad_g, grad_b, static_cast<double*>(scratch), grad_params,
                                  reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "fit adjoint");
    write_error(error, "");
    return ok_status();
}


// ---- spatial DIR (carrier input) ----

static FjStatus spatial_check(FjbRecipe* recipe, const FjbFitParams* params, const float* cb, const float* cg,
                              const float* cr, ptrdiff_t stride, int32_t width, int32_t height, fjb::FitTheta& th,
                              FjErrorBuffer* error) {
    FjStatus st = fit_check(recipe, params, cb && cg && cr, 3, width, height, th, error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (recipe->r.params.dir_mode == fjb::kDirInactive)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "spatial DIR fitting needs active DIR couplers");
    if (stride < width) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "carrier stride below the width");
    return ok_status();
}

FjStatus fjb_fit_dir_source_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                    const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                    float* corr_y, float* corr_m, float* corr_c, int32_t width, int32_t height,
                                    void* stream, FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = spatial_check(recipe, params, carrier_b, carrier_g, carrier_r, carrier_stride, width, height, th,
                                error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!corr_y || !corr_m || !corr_c) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if ((long long)width * height > 0) {
        fjb::PixelParams p = recipe->r.params;
        p.width = width;
        p.height = height;
        const fjb::FitCarrier cr{carrier_b, carrier_g, carrier_r, (long long)carrier_stride, nullptr, nullptr, nullptr};
        const cudaError_t e =
            fjb::launch_fit_dir_source(p, th, cr, corr_y, corr_m, corr_c, reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_status(e, error, "fit DIR source");
    }
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_fit_forward_spatial_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                         const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                         const float* filtered_y, const float* filtered_m, const float* filtered_c,
                                         float* out_r, float* out_g, float* out_b, int32_t width, int32_t height,
                                         void* stream, FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = spatial_check(recipe, params, carrier_b, carrier_g, carrier_r, carrier_stride, width, height, th,
                                error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!out_r || !out_g || !out_b || !filtered_y || !filtered_m || !filtered_c)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if ((long long)width * height > 0) {
        fjb::PixelParams p = recipe->r.params;
        p.width = width;
        p.height = height;
        fjb::FitCarrier cr{carrier_b, carrier_g, carrier_r, (long long)carrier_stride, nullptr, nullptr, nullptr};
        cr.fy = filtered_y;
        cr.fm = filtered_m;
        cr.fc = filtered_c;
        const cudaError_t e = fjb::launch_fit_forward<true, true>(p, th, cr, out_r, out_g, out_b,
                                                                  reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_status(e, error, "fit forward");
    }
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_fit_vjp_spatial_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                     const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                     const float* filtered_y, const float* filtered_m, const float* filtered_c,
                                     const float* grad_r, const float* grad_g, const float* grad_b, int32_t width,
                                     int32_t height, double* grad_params, float* grad_carrier_b, float* grad_carrier_g,
                                     float* grad_carrier_r, float* grad_filtered_y, float* grad_filtered_m,
                                     float* grad_filtered_c, void* scratch, size_t scratch_bytes, void* stream,
                                     FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = spatial_check(recipe, params, carrier_b, carrier_g, carrier_r, carrier_stride, width, height, th,
                                error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!grad_r || !grad_g || !grad_b || !grad_params || !scratch || !filtered_y || !filtered_m || !filtered_c ||
        !grad_filtered_y || !grad_filtered_m || !grad_filtered_c)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    const bool planes = grad_carrier_b || grad_carrier_g || grad_carrier_r;
    if (planes && !(grad_carrier_b && grad_carrier_g && grad_carrier_r))
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "carrier gradient planes: all three or none");
    if (scratch_bytes < (size_t)fjb::fit_blocks() * fjb::kFitParams * sizeof(double))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "fit scratch smaller than fjb_fit_scratch_bytes()");
    fjb::PixelParams p = recipe->r.params;
    p.width = width;
    p.height = height;
    fjb::FitCarrier cr{carrier_b,      carrier_g,      carrier_r,     (long long)carrier_stride,
                       grad_carrier_b, grad_carrier_g, grad_carrier_r};
    cr.fy = filtered_y;
    cr.fm = filtered_m;
    cr.fc = filtered_c;
    cr.gfy = grad_filtered_y;
    cr.gfm = grad_filtered_m;
    cr.gfc = grad_filtered_c;
    const cudaError_t e =
        fjb::launch_fit_vjp<true, true>(p, th, cr, grad_r, grad_g, grad_b, static_cast<double*>(scratch), grad_params,
                                        reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "fit adjoint");
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_fit_dir_source_vjp_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                        const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                        const float* grad_corr_y, const float* grad_corr_m, const float* grad_corr_c,
                                        int32_t width, int32_t height, double* grad_params, float* grad_carrier_b,
                                        float* grad_carrier_g, float* grad_carrier_r, void* scratch,
                                        size_t scratch_bytes, void* stream, FjErrorBuffer* error) {
    fjb::FitTheta th{};
    FjStatus st = spatial_check(recipe, params, carrier_b, carrier_g, carrier_r, carrier_stride, width, height, th,
                                error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (!grad_corr_y || !grad_corr_m || !grad_corr_c || !grad_params || !scratch)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    const bool planes = grad_carrier_b || grad_carrier_g || grad_carrier_r;
    if (planes && !(grad_carrier_b && grad_carrier_g && grad_carrier_r))
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "carrier gradient planes: all three or none");
    if (scratch_bytes < (size_t)fjb::fit_blocks() * fjb::kFitParams * sizeof(double))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "fit scratch smaller than fjb_fit_scratch_bytes()");
    fjb::PixelParams p = recipe->r.params;
    p.width = width;
    p.height = height;
    const fjb::FitCarrier cr{carrier_b,      carrier_g,      carrier_r,     (long long)carrier_stride,
                             grad_carrier_b, grad_carrier_g, grad_carrier_r};
    const cudaError_t e = fjb::launch_fit_dir_source_vjp(p, th, cr, grad_corr_y, grad_corr_m, grad_corr_c,
                                                         static_cast<double*>(scratch), grad_params,
                                                         reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "fit DIR source adjoint");
    write_error(error, "");
    return ok_status();
}

} // extern "C"
