/* oracle.c -- CPU restatement of Film-Juicer's per-pixel render chain (TEST ORACLE).
 *
 * This file is test infrastructure. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it, and only as the checker or the
 * timed CPU baseline; the product (libjuicer_b200.so) never calls it.
 *
 * It restates, in plain C with no fused multiply-add (built with -ffp-contract=off),
 * the reference's device math for the render path, step by step, and the reference's
 * host packing of FjPreparedHostData into kernel payloads. Each function cites the
 * reference file:line it follows. Scalar FP32/FP64 choices follow the reference:
 * FP32 for exposure, curves, DIR, print and LUT interpolation; FP64 for the scan
 * normalisation, scanner colour matrices and the output encoding; the scanner LUT
 * build is FP64 (rust/film-juicer-core/src/scanner/lut.rs). libm's expf/log10f/...
 * replace CUDA's device functions, so FP32 results may differ from a GPU in the
 * last bits; integer work (interval searches, LUT cells, failure masks) is exact.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/juicer_b200.h"
#include "../include/juicer_cuda_api.h"

#define NL 81
#define TC 192

typedef struct {
    const float* x;
    const float* y; /* strided */
    int ystride;
    int n;
} Curve;

typedef struct {
    /* film */
    int method, input_cs, decode, adapt;
    float m_rgb_xyz[9], m_adapt[9], m_xyz_srgb[9];
    const float* tc; /* [192][192][4] */
    const float* mallett_basis;
    const float* mallett_illum;
    float sens_bgr[3][NL];
    float mallett_midgray;
    float manual, route;
    float gamma_bgr[3];
    int dir_mode;
    float M[9], dmax[3], dref[3], dk[3], rcref[3], rkr[3];
    Curve dens[3], dirc[3];
    /* print */
    int print;
    const float *eps_c_src, *base_src, *pillum, *psens; /* strided [81][3] */
    float print_exposure, print_route, preflash, midgray, preflash_raw[3];
    Curve pdc[3];
    /* scan */
    int medium_negative;
    float min_cmy[3], inv_cmy[3];
    int res;
    float *lut_v, *lut_sc, *lut_sm, *lut_sy, *cell_lo, *cell_hi;
    int corr_active;
    float corr_slope, corr_offset;
    float cat02[9], xyz_rgb[9], illum_xyz[3];
    int gamut;
    const float* cmax;
    float g_to_xyz[9], g_from_xyz[9], lknee[3], cknee[3];
    int enc_iso, enc_cctf;
    float dwg[9];
    int cctf_kind;
    float cg, ca, cb, cc, cd, ccut;
} Pack;

/* ---------------- scanner LUT (rust/film-juicer-core/src/scanner/lut.rs:108-296) ---------------- */

static void pchip_slopes(const double* v, int n, double* out, double* d) {
    for (int i = 0; i < n - 1; ++i) d[i] = v[i + 1] - v[i];
    if (n == 2) {
        out[0] = out[1] = d[0];
        return;
    }
#define ENDPOINT(a, b, res)                                                          \
    do {                                                                             \
        double s_ = 0.5 * (3.0 * (a) - (b));                                         \
        if (s_ * (a) <= 0.0) res = 0.0;                                              \
        else if ((a) * (b) < 0.0 && fabs(s_) > fabs(3.0 * (a))) res = 3.0 * (a);     \
        else res = s_;                                                               \
    } while (0)
    ENDPOINT(d[0], d[1], out[0]);
    for (int i = 1; i < n - 1; ++i) {
        double p = d[i - 1], q = d[i];
        out[i] = (p == 0.0 || q == 0.0 || p * q <= 0.0) ? 0.0 : 2.0 * p * q / (p + q);
    }
    ENDPOINT(d[n - 2], d[n - 3], out[n - 1]);
#undef ENDPOINT
}

/* Returns 0 on success, 1 when a node is not finite. */
int oracle_scanner_lut(const FjbScannerLutInput* in, float* log2_xyz, float* sc, float* sm, float* sy, float* cmin,
                       float* cmax) {
    const int r = (int)in->resolution;
    const int k = in->sample_count;
    if (r < 2) return 2;
    const size_t count = (size_t)r * r * r * 3;
    double* nodes = (double*)malloc(count * sizeof(double));
    double* line = (double*)malloc((size_t)r * sizeof(double));
    double* lsl = (double*)malloc((size_t)r * sizeof(double));
    double* del = (double*)malloc((size_t)r * sizeof(double));
    int fail = 0;
    for (int c = 0; c < r && !fail; ++c)
        for (int m = 0; m < r && !fail; ++m)
            for (int y = 0; y < r && !fail; ++y) {
                const int idx[3] = {c, m, y};
                double dens[3];
                for (int ch = 0; ch < 3; ++ch) {
                    double nrm = (double)idx[ch] / (double)(r - 1);
                    double scaled = nrm / (double)in->inverse_span_cmy[ch];
                    dens[ch] = in->medium == 0 ? scaled - (double)in->range_min_cmy[ch]
                                               : scaled + (double)in->range_min_cmy[ch];
                }
                double xyz[3] = {0, 0, 0};
                const float* w[3] = {in->weighted_x.data, in->weighted_y.data, in->weighted_z.data};
                for (int s = 0; s < k; ++s) {
                    double base = in->has_baseline ? (double)in->baseline_min.data[s] : 0.0;
                    double spectral = dens[0] * (double)in->eps_c.data[s] + dens[1] * (double)in->eps_m.data[s] +
                                      dens[2] * (double)in->eps_y.data[s] + base;
                    double t = pow(10.0, -spectral);
                    for (int ch = 0; ch < 3; ++ch) {
                        double wk = (double)w[ch][s];
                        if (isfinite(wk)) {
                            double p = t * wk;
                            if (!isnan(p)) xyz[ch] += p;
                        }
                    }
                }
                for (int ch = 0; ch < 3; ++ch) {
                    double sum = xyz[ch] * (double)in->inv_yn;
                    double lg = log10(fmax(sum, 0.0) + 1e-10);
                    if (!isfinite(lg)) fail = 1;
                    size_t i = ((((size_t)c * r + m) * r + y) * 3) + ch;
                    nodes[i] = lg * 3.32192809488736234787;
                    log2_xyz[i] = (float)nodes[i];
                }
            }
    if (!fail) {
        float* outs[3] = {sc, sm, sy};
        for (int axis = 0; axis < 3; ++axis)
            for (int a = 0; a < r; ++a)
                for (int b = 0; b < r; ++b)
                    for (int ch = 0; ch < 3; ++ch) {
                        for (int i = 0; i < r; ++i) {
                            int cc = axis == 0 ? i : a, mm = axis == 0 ? a : (axis == 1 ? i : b),
                                yy = axis == 2 ? i : b;
                            line[i] = nodes[((((size_t)cc * r + mm) * r + yy) * 3) + ch];
                        }
                        pchip_slopes(line, r, lsl, del);
                        for (int i = 0; i < r; ++i) {
                            int cc = axis == 0 ? i : a, mm = axis == 0 ? a : (axis == 1 ? i : b),
                                yy = axis == 2 ? i : b;
                            outs[axis][((((size_t)cc * r + mm) * r + yy) * 3) + ch] = (float)lsl[i];
                        }
                    }
        const int s = r - 1;
        for (int c = 0; c < s; ++c)
            for (int m = 0; m < s; ++m)
                for (int y = 0; y < s; ++y)
                    for (int ch = 0; ch < 3; ++ch) {
                        double lo = nodes[((((size_t)c * r + m) * r + y) * 3) + ch], hi = lo;
                        for (int dc = 0; dc < 2; ++dc)
                            for (int dm = 0; dm < 2; ++dm)
                                for (int dy = 0; dy < 2; ++dy) {
                                    double v = nodes[((((size_t)(c + dc) * r + (m + dm)) * r + (y + dy)) * 3) + ch];
                                    if (v < lo) lo = v;
                                    if (hi < v) hi = v;
                                }
                        size_t i = ((((size_t)c * s + m) * s + y) * 3) + ch;
                        cmin[i] = (float)lo;
                        cmax[i] = (float)hi;
                    }
    }
    free(nodes);
    free(line);
    free(lsl);
    free(del);
    return fail;
}

/* ---------------- device math (src/Cuda/JuicerCudaDeviceHelpers.cuh) ---------------- */

static float keepf(float v) { return isfinite(v) ? v : 0.0f; }

static void mat3(const float* m, const float* v, float* o) {
    o[0] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    o[1] = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    o[2] = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
}

static void mat3d(const float* m, const double* v, double* o) {
    o[0] = (double)m[0] * v[0] + (double)m[1] * v[1] + (double)m[2] * v[2];
    o[1] = (double)m[3] * v[0] + (double)m[4] * v[1] + (double)m[5] * v[2];
    o[2] = (double)m[6] * v[0] + (double)m[7] * v[1] + (double)m[8] * v[2];
}

/* :175-196 */
static float dec_bt2020(float v) {
    float x = fmaxf(0.0f, keepf(v));
    const float a = 1.09929681f;
    if (x < 0.0812428791f) return x / 4.5f;
    return powf((x + (a - 1.0f)) / a, 1.0f / 0.45f);
}
static float dec_srgb(float v) {
    float x = fmaxf(0.0f, keepf(v));
    if (x <= 0.04045f) return x / 12.92f;
    return powf((x + 0.055f) / 1.055f, 2.4f);
}
/* :198-225 */
static void decode(const Pack* p, const float* in, float* out) {
    for (int c = 0; c < 3; ++c) {
        if (p->decode && p->input_cs == 1) out[c] = dec_bt2020(in[c]);
        else if (p->decode && p->input_cs == 3) out[c] = dec_srgb(in[c]);
        else out[c] = keepf(in[c]);
    }
}

/* :254-275 */
static float mitchell(float t) {
    const float B = 1.0f / 3.0f, C = 1.0f / 3.0f;
    float x = fabsf(t);
    if (x < 1.0f)
        return (1.0f / 6.0f) * ((12.0f - 9.0f * B - 6.0f * C) * x * x * x + (-18.0f + 12.0f * B + 6.0f * C) * x * x +
                                (6.0f - 2.0f * B));
    if (x < 2.0f)
        return (1.0f / 6.0f) * ((-B - 6.0f * C) * x * x * x + (6.0f * B + 30.0f * C) * x * x +
                                (-12.0f * B - 48.0f * C) * x + (8.0f * B + 24.0f * C));
    return 0.0f;
}
/* :277-289 */
static void tc_coord(float nrm, int* base, float* frac) {
    float coord = fminf(1.0f, fmaxf(0.0f, nrm)) * (float)(TC - 1);
    if (coord >= (float)(TC - 1)) {
        *base = TC - 2;
        *frac = 1.0f;
        return;
    }
    *base = (int)floorf(coord);
    *frac = coord - (float)*base;
}
static int reflect(int i) {
    if (i < 0) return -i;
    if (i >= TC) return 2 * (TC - 1) - i;
    return i;
}
/* :291-327 */
static float tc_sample(const float* lut, int ch, float qc, float qm) {
    int cb, mb;
    float cf, mf;
    tc_coord(qc, &cb, &cf);
    tc_coord(qm, &mb, &mf);
    float wc[4] = {mitchell(cf + 1.0f), mitchell(cf), mitchell(cf - 1.0f), mitchell(cf - 2.0f)};
    float wm[4] = {mitchell(mf + 1.0f), mitchell(mf), mitchell(mf - 1.0f), mitchell(mf - 2.0f)};
    float v = 0.0f, ws = 0.0f;
    for (int dc = 0; dc < 4; ++dc) {
        int c = reflect(cb - 1 + dc);
        for (int dm = 0; dm < 4; ++dm) {
            int m = reflect(mb - 1 + dm);
            float w = wc[dc] * wm[dm];
            ws += w;
            v += w * lut[((size_t)c * TC + m) * 4 + ch];
        }
    }
    return ws != 0.0f ? v / ws : 0.0f;
}

/* :537-617 */
static void tc_exposure(const Pack* p, const float* in, float* e) {
    float lin[3], xyz[3], w[3];
    decode(p, in, lin);
    mat3(p->m_rgb_xyz, lin, xyz);
    if (p->adapt) mat3(p->m_adapt, xyz, w);
    else memcpy(w, xyz, sizeof(w));
    for (int c = 0; c < 3; ++c) w[c] = keepf(w[c]);
    float X = keepf(w[0]), Y = keepf(w[1]), Z = keepf(w[2]);
    float sum = X + Y + Z;
    float den = fmaxf(sum, 1e-10f);
    float x = X / den, y = Y / den;
    float qd = fmaxf(1.0f - x, 1e-10f);
    float qx = (1.0f - x);
    qx = qx * qx;
    float qy = y / qd;
    qx = fminf(1.0f, fmaxf(0.0f, qx));
    qy = fminf(1.0f, fmaxf(0.0f, qy));
    float r = tc_sample(p->tc, 0, qx, qy), g = tc_sample(p->tc, 1, qx, qy), b = tc_sample(p->tc, 2, qx, qy);
    e[0] = keepf(sum * keepf(b));
    e[1] = keepf(sum * keepf(g));
    e[2] = keepf(sum * keepf(r));
}

/* :509-535, :619-668 */
static void mallett_exposure(const Pack* p, const float* in, float* e) {
    float lin[3], xyz[3], ad[3], s[3];
    decode(p, in, lin);
    mat3(p->m_rgb_xyz, lin, xyz);
    const float* src = xyz;
    if (p->adapt) {
        mat3(p->m_adapt, xyz, ad);
        src = ad;
    }
    mat3(p->m_xyz_srgb, src, s);
    for (int c = 0; c < 3; ++c) s[c] = keepf(s[c]);
    float r = fmaxf(0.0f, keepf(s[0])), g = fmaxf(0.0f, keepf(s[1])), b = fmaxf(0.0f, keepf(s[2]));
    float eb = 0, eg = 0, er = 0;
    for (int i = 0; i < NL; ++i) {
        float il = p->mallett_illum[i];
        float spd = (r * p->mallett_basis[3 * i] + g * p->mallett_basis[3 * i + 1] + b * p->mallett_basis[3 * i + 2]) * il;
        if (!isfinite(spd)) continue;
        if (isfinite(p->sens_bgr[0][i])) eb += spd * p->sens_bgr[0][i];
        if (isfinite(p->sens_bgr[1][i])) eg += spd * p->sens_bgr[1][i];
        if (isfinite(p->sens_bgr[2][i])) er += spd * p->sens_bgr[2][i];
    }
    e[0] = isfinite(eb) ? fmaxf(0.0f, eb) : 0.0f;
    e[1] = isfinite(eg) ? fmaxf(0.0f, eg) : 0.0f;
    e[2] = isfinite(er) ? fmaxf(0.0f, er) : 0.0f;
    for (int c = 0; c < 3; ++c) e[c] = fmaxf(0.0f, e[c] * p->mallett_midgray);
}

/* :710-736 */
static void film_exposure(const Pack* p, const float* in, float ae, int with_route, float* e) {
    if (p->method == FJ_RAW_MALLETT_2019) mallett_exposure(p, in, e);
    else tc_exposure(p, in, e);
    float a = 1.0f;
    if (isfinite(ae) && ae > 0.0f) a = ae;
    float s = a * p->manual;
    if (with_route) s *= p->route;
    s = (isfinite(s) && s > 0.0f) ? s : 1.0f;
    for (int c = 0; c < 3; ++c) e[c] = fmaxf(0.0f, e[c] * s);
}

/* :34-89 */
static float curve_at(const Curve* c, float logE, float gamma) {
    if (!isfinite(logE)) return nanf("");
    float xq = logE * gamma;
    int last = c->n - 1;
    float xmin = c->x[0], xmax = c->x[last];
    if (!(xmax >= xmin)) return c->y[0];
    if (xq <= xmin) return c->y[0];
    if (xq >= xmax) return c->y[(size_t)last * c->ystride];
    int lo = 1, hi = last, i1 = last + 1;
    while (lo <= hi) {
        int mid = lo + ((hi - lo) >> 1);
        if (xq < c->x[mid]) {
            i1 = mid;
            hi = mid - 1;
        } else lo = mid + 1;
    }
    if (i1 > last) return c->y[(size_t)last * c->ystride];
    int i0 = i1 - 1;
    float x0 = c->x[i0], x1 = c->x[i1], y0 = c->y[(size_t)i0 * c->ystride], y1 = c->y[(size_t)i1 * c->ystride];
    float den = x1 - x0;
    if (!(den > 0.0f) || !isfinite(den)) return y0;
    float t = (xq - x0) / den;
    return y0 + t * (y1 - y0);
}
/* :91-105 */
static float inf_clamp(const Curve* c, float logE) {
    if (isfinite(logE) || isnan(logE)) return logE;
    float xmin = c->x[0], xmax = c->x[c->n - 1];
    if (!(xmax >= xmin)) return logE;
    return logE > 0.0f ? xmax : xmin;
}

/* :1073-1123 */
static int langmuir(float v, float k, float ref, float* out) {
    *out = nanf("");
    if (!isfinite(v) || !isfinite(k) || !(k > 0.0f) || !isfinite(ref)) return 0;
    float den = k + v, kr = k + ref;
    int direct = isfinite(den) && den != 0.0f && isfinite(kr) && (v == 0.0f || fabsf(v) <= FLT_MAX / fabsf(kr));
    if (direct) {
        *out = v * kr / den;
        return isfinite(*out);
    }
    float ns = 1.0f + ref / k;
    if (!isfinite(ns)) return 0;
    if (v >= 0.0f) {
        float ds = 1.0f + v / k;
        if (!isfinite(ds) || ds == 0.0f) return 0;
        *out = (v / ds) * ns;
        return isfinite(*out);
    }
    if (!isfinite(den) || den == 0.0f) return 0;
    float ds = den / k;
    if (!isfinite(ds) || ds == 0.0f) return 0;
    if (fabsf(v) <= FLT_MAX / fabsf(ns)) *out = v * ns / ds;
    else *out = (v / ds) * ns;
    return isfinite(*out);
}

/* :1125-1241 */
static unsigned dir_runtime(const Pack* p, float* logE, const float* layer) {
    float donor[3] = {p->dmax[0] - layer[0], p->dmax[1] - layer[1], p->dmax[2] - layer[2]};
    unsigned fail = 0;
    if (p->dir_mode == FJ_DIR_NEGATIVE_DONOR_LANGMUIR)
        for (int c = 0; c < 3; ++c)
            if (!langmuir(layer[c], p->dk[c], p->dref[c], &donor[c])) fail |= 1u << c;
    float corr[3];
    corr[0] = p->M[0] * donor[0] + p->M[3] * donor[1] + p->M[6] * donor[2];
    corr[1] = p->M[1] * donor[0] + p->M[4] * donor[1] + p->M[7] * donor[2];
    corr[2] = p->M[2] * donor[0] + p->M[5] * donor[1] + p->M[8] * donor[2];
    for (int c = 0; c < 3; ++c)
        if (!isfinite(corr[c])) fail |= 1u << c;
    if (p->dir_mode == FJ_DIR_POSITIVE_RECEIVER_LANGMUIR) {
        for (int c = 0; c < 3; ++c) {
            if (p->rcref[c] == 0.0f) {
                corr[c] = 0.0f;
                continue;
            }
            float v = corr[c];
            if (!langmuir(v, p->rkr[c], p->rcref[c], &corr[c])) fail |= 1u << c;
        }
    }
    if (fail) return fail;
    unsigned sf = 0;
    for (int c = 0; c < 3; ++c) {
        float o = logE[c];
        if (isnan(o)) {
            sf |= 1u << c;
            continue;
        }
        logE[c] = o - corr[c];
        if ((!isinf(o) && !isfinite(logE[c])) || (isinf(o) && (!isinf(logE[c]) || signbit(o) != signbit(logE[c]))))
            sf |= 1u << c;
    }
    return sf;
}

/* src/Cuda/Scan/JuicerCudaScanPipeline.cu:1622-1698 with :766-846 of the helpers */
static unsigned capture_density(const Pack* p, const float* e_in, float* d) {
    float logE[3], logS[3], layer[3];
    for (int c = 0; c < 3; ++c) {
        logE[c] = log10f(fmaxf(e_in[c], 0.0f) + 1e-10f);
        logS[c] = inf_clamp(&p->dens[c], logE[c]);
        layer[c] = curve_at(&p->dens[c], logS[c], p->gamma_bgr[c]);
    }
    if (p->dir_mode == FJ_DIR_INACTIVE) {
        d[0] = layer[2];
        d[1] = layer[1];
        d[2] = layer[0];
        return 0;
    }
    float lc[3] = {logS[0], logS[1], logS[2]};
    unsigned f = dir_runtime(p, lc, layer);
    if (f) {
        d[0] = d[1] = d[2] = nanf("");
        return f;
    }
    d[2] = curve_at(&p->dirc[0], lc[0], p->gamma_bgr[0]);
    d[1] = curve_at(&p->dirc[1], lc[1], p->gamma_bgr[1]);
    d[0] = curve_at(&p->dirc[2], lc[2], p->gamma_bgr[2]);
    return 0;
}

/* :866-1071 (FP32, same accumulation order as the reference loop) */
/* The print's spectral integral raw_c = sum_l 10^-D(l) I(l) S_c(l) with the reference's
 * NaN-sensitivity skips (src/Cuda/JuicerCudaDeviceHelpers.cuh:866-933). */
static void print_spectral_raw(const Pack* p, const float* D, float raw[3]) {
    float ac = 0, am = 0, ay = 0;
    for (int i = 0; i < NL; ++i) {
        float sC = p->psens[i * 3], sM = p->psens[i * 3 + 1], sY = p->psens[i * 3 + 2];
        int aC = !isnan(sC), aM = !isnan(sM), aY = !isnan(sY);
        if (!aC && !aM && !aY) continue;
        float base = p->base_src[i];
        float ds = D[0] * p->eps_c_src[i * 3] + D[1] * p->eps_c_src[i * 3 + 1] + D[2] * p->eps_c_src[i * 3 + 2] + base;
        float t = exp2f(-ds * 3.32192809488736234787f) * p->pillum[i];
        float e = isnan(t) ? 0.0f : t;
        if (aC) ac += e * sC;
        if (aM) am += e * sM;
        if (aY) ay += e * sY;
    }
    raw[0] = ac;
    raw[1] = am;
    raw[2] = ay;
}

static void print_stage_dust(const Pack* p, float* D, float dust);
static void print_stage(const Pack* p, float* D) { print_stage_dust(p, D, 1.0f); }

/* src/Cuda/JuicerCudaDeviceHelpers.cuh:1047-1070: `dust` scales the spectral raw print
 * exposure before the exposure scales */
static void print_stage_dust(const Pack* p, float* D, float dust) {
    float raw[3];
    print_spectral_raw(p, D, raw);
    if (dust != 1.0f)
        for (int c = 0; c < 3; ++c) raw[c] *= dust;
    for (int c = 0; c < 3; ++c) raw[c] *= p->midgray;
    if (isfinite(p->preflash) && p->preflash > 0.0f)
        for (int c = 0; c < 3; ++c) raw[c] += p->preflash_raw[c] * p->preflash;
    for (int c = 0; c < 3; ++c) raw[c] *= p->print_exposure;
    for (int c = 0; c < 3; ++c) raw[c] *= p->print_route;
    for (int c = 0; c < 3; ++c) D[c] = curve_at(&p->pdc[c], log10f(raw[c] + 1e-10f), 1.0f);
}

/* :357-506 */
static void pchip_coord(float nrm, int res, int* base, float* frac) {
    float coord = nrm * (float)(res - 1);
    coord = fminf((float)(res - 1), fmaxf(0.0f, coord));
    if (coord >= (float)(res - 1)) {
        *base = res - 2;
        *frac = 1.0f;
        return;
    }
    *base = (int)floorf(coord);
    *frac = coord - (float)*base;
}
static float herm(float y0, float y1, float m0, float m1, float t) {
    float t2 = t * t, t3 = t2 * t;
    float h00 = 2.0f * t3 - 3.0f * t2 + 1.0f, h10 = t3 - 2.0f * t2 + t, h01 = -2.0f * t3 + 3.0f * t2, h11 = t3 - t2;
    return h00 * y0 + h10 * m0 + h01 * y1 + h11 * m1;
}
static float lmix(float a, float b, float t) { return a + t * (b - a); }

static int scan_lut(const Pack* p, const double* n, float* out) {
    if (!isfinite(n[0]) || !isfinite(n[1]) || !isfinite(n[2])) return 0;
    int r = p->res, c, m, y;
    float tc, tm, ty;
    pchip_coord((float)n[0], r, &c, &tc);
    pchip_coord((float)n[1], r, &m, &tm);
    pchip_coord((float)n[2], r, &y, &ty);
#define AT(T, cc, mm, yy, o) (T)[((((size_t)(cc) * r + (mm)) * r + (yy)) * 3) + (o)]
    for (int o = 0; o < 3; ++o) {
        float v000 = herm(AT(p->lut_v, c, m, y, o), AT(p->lut_v, c + 1, m, y, o), AT(p->lut_sc, c, m, y, o),
                          AT(p->lut_sc, c + 1, m, y, o), tc);
        float v010 = herm(AT(p->lut_v, c, m + 1, y, o), AT(p->lut_v, c + 1, m + 1, y, o),
                          AT(p->lut_sc, c, m + 1, y, o), AT(p->lut_sc, c + 1, m + 1, y, o), tc);
        float v001 = herm(AT(p->lut_v, c, m, y + 1, o), AT(p->lut_v, c + 1, m, y + 1, o),
                          AT(p->lut_sc, c, m, y + 1, o), AT(p->lut_sc, c + 1, m, y + 1, o), tc);
        float v011 = herm(AT(p->lut_v, c, m + 1, y + 1, o), AT(p->lut_v, c + 1, m + 1, y + 1, o),
                          AT(p->lut_sc, c, m + 1, y + 1, o), AT(p->lut_sc, c + 1, m + 1, y + 1, o), tc);
        float sm00 = lmix(AT(p->lut_sm, c, m, y, o), AT(p->lut_sm, c + 1, m, y, o), tc);
        float sm10 = lmix(AT(p->lut_sm, c, m + 1, y, o), AT(p->lut_sm, c + 1, m + 1, y, o), tc);
        float sm01 = lmix(AT(p->lut_sm, c, m, y + 1, o), AT(p->lut_sm, c + 1, m, y + 1, o), tc);
        float sm11 = lmix(AT(p->lut_sm, c, m + 1, y + 1, o), AT(p->lut_sm, c + 1, m + 1, y + 1, o), tc);
        float vy0 = herm(v000, v010, sm00, sm10, tm);
        float vy1 = herm(v001, v011, sm01, sm11, tm);
        float sy0 = lmix(lmix(AT(p->lut_sy, c, m, y, o), AT(p->lut_sy, c + 1, m, y, o), tc),
                         lmix(AT(p->lut_sy, c, m + 1, y, o), AT(p->lut_sy, c + 1, m + 1, y, o), tc), tm);
        float sy1 = lmix(lmix(AT(p->lut_sy, c, m, y + 1, o), AT(p->lut_sy, c + 1, m, y + 1, o), tc),
                         lmix(AT(p->lut_sy, c, m + 1, y + 1, o), AT(p->lut_sy, c + 1, m + 1, y + 1, o), tc), tm);
        float v = herm(vy0, vy1, sy0, sy1, ty);
        int s = r - 1;
        size_t ci = ((((size_t)c * s + m) * s + y) * 3) + o;
        out[o] = fminf(p->cell_hi[ci], fmaxf(p->cell_lo[ci], v));
    }
#undef AT
    return 1;
}

/* src/GamutCompression.h:110-216 */
static const float OK_XL[9] = {0.8189330101f, 0.3618667424f, -0.1288597137f, 0.0329845436f, 0.9293118715f,
                               0.0361456387f, 0.0482003018f, 0.2643662691f, 0.6338517070f};
static const float OK_LX[9] = {1.2270138511f,  -0.5577999807f, 0.2812561490f,  -0.0405801784f, 1.1122568696f,
                               -0.0716766787f, -0.0763812845f, -0.4214819784f, 1.5861632204f};
static const float OK_RL[9] = {0.2104542553f, 0.7936177850f, -0.0040720468f, 1.9779984951f, -2.4285922050f,
                               0.4505937099f, 0.0259040371f, 0.7827717662f, -0.8086757660f};
static const float OK_LR[9] = {1.0f, 0.3963377774f,  0.2158037573f,  1.0f, -0.1055613458f,
                               -0.0638541728f, 1.0f, -0.0894841775f, -1.2914855480f};
static float scbrt(float v) { return v < 0.0f ? -cbrtf(-v) : cbrtf(v); }
static float knee(float v, const float* k) {
    if (!(v > k[0])) return v;
    float span = k[1] - k[0], nrm = (v - k[0]) / span;
    return k[0] + span * nrm / powf(1.0f + powf(nrm, k[2]), 1.0f / k[2]);
}
static float boundary(const float* cmax, float L, float h) {
    const float PI = 3.14159265358979323846f, TWO_PI = 2.0f * PI;
    float Lc = fminf(fmaxf(L, 0.02f), 1.0f);
    float lp = (Lc - 0.02f) / (1.0f - 0.02f) * 63.0f;
    int l0 = (int)floorf(lp), l1 = l0 + 1 < 64 ? l0 + 1 : l0;
    float lf = lp - (float)l0;
    float wh = fmodf(h + PI, TWO_PI);
    if (wh < 0.0f) wh += TWO_PI;
    float hp = wh / TWO_PI * 720.0f;
    int h0 = (int)floorf(hp) % 720, h1 = (h0 + 1) % 720;
    float hf = hp - floorf(hp);
    int r0 = l0 * 720, r1 = l1 * 720;
    float a = cmax[r0 + h0] + hf * (cmax[r0 + h1] - cmax[r0 + h0]);
    float b = cmax[r1 + h0] + hf * (cmax[r1 + h1] - cmax[r1 + h0]);
    return a + lf * (b - a);
}
static void gamut(const Pack* p, float* rgb) {
    float xyz[3], lms[3], lab[3];
    mat3(p->g_to_xyz, rgb, xyz);
    mat3(OK_XL, xyz, lms);
    for (int c = 0; c < 3; ++c) lms[c] = scbrt(lms[c]);
    mat3(OK_RL, lms, lab);
    lab[0] = knee(lab[0], p->lknee);
    float ch = hypotf(lab[1], lab[2]);
    if (ch > 0.0f) {
        float hue = atan2f(lab[2], lab[1]);
        float b = fmaxf(boundary(p->cmax, lab[0], hue), 1.0e-9f);
        float cmp = knee(ch / b, p->cknee) * b;
        float s = cmp / ch;
        lab[1] *= s;
        lab[2] *= s;
    }
    mat3(OK_LR, lab, lms);
    for (int c = 0; c < 3; ++c) lms[c] = lms[c] * lms[c] * lms[c];
    mat3(OK_LX, lms, xyz);
    mat3(p->g_from_xyz, xyz, rgb);
}

/* src/Cuda/Scan/JuicerCudaScanPipeline.cu:99-192 */
static double clamp01(double v) { return v <= 0.0 ? 0.0 : (v >= 1.0 ? 1.0 : v); }
static float enc(const Pack* p, float v) {
    switch (p->cctf_kind) {
        case 0: return v;
        case 1: return copysignf(powf(fabsf(v), p->cg), v);
        case 2: return v <= 0.0031308f ? 12.92f * v : 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
        case 3: return v < p->cb ? v * 4.5f : p->ca * powf(v, 0.45f) - (p->ca - 1.0f);
        case 4: return v < p->ccut ? v * 16.0f : powf(v, p->cg);
        case 5: {
            float l = fmaxf(0.0f, v);
            return l <= p->ccut ? l * p->cd : (log2f(l + p->ca) + p->cb) * p->cc;
        }
        default: return (float)clamp01(v);
    }
}

/* :1700-1840, :1944-2037: density -> linear output RGB (glare percent added in XYZ when
 * glare >= 0); returns 0 on a scan failure */
static int scan_lin_dust(const Pack* p, const float* D, double* rgb, float glare, const float* dust);
static int scan_lin(const Pack* p, const float* D, double* rgb, float glare) { return scan_lin_dust(p, D, rgb, glare, NULL); }

/* `dust`: film dust transmittance scaling the scanned XYZ (direct route, :2006-2011) */
static int scan_lin_dust(const Pack* p, const float* D, double* rgb, float glare, const float* dust) {
    double n[3];
    for (int c = 0; c < 3; ++c)
        n[c] = p->medium_negative ? ((double)D[c] + (double)p->min_cmy[c]) * (double)p->inv_cmy[c]
                                  : ((double)D[c] - (double)p->min_cmy[c]) * (double)p->inv_cmy[c];
    float l2[3];
    if (!scan_lut(p, n, l2)) return 0;
    double xyz[3] = {(double)exp2f(l2[0]), (double)exp2f(l2[1]), (double)exp2f(l2[2])};
    if (dust)
        for (int c = 0; c < 3; ++c) xyz[c] *= (double)*dust;
    if (p->corr_active) {
        double cy = fmin(fmax((double)p->corr_slope * xyz[1] + (double)p->corr_offset, 0.0), 1.0);
        double s = cy / (xyz[1] + 1e-10);
        for (int c = 0; c < 3; ++c) xyz[c] *= s;
    }
    if (glare >= 0.0f) {
        double g = (double)glare * 0.01;
        for (int c = 0; c < 3; ++c) xyz[c] += g * (double)p->illum_xyz[c];
    }
    double ad[3];
    mat3d(p->cat02, xyz, ad);
    mat3d(p->xyz_rgb, ad, rgb);
    if (!isfinite(rgb[0]) || !isfinite(rgb[1]) || !isfinite(rgb[2])) return 0;
    if (p->gamut) {
        float f[3] = {(float)rgb[0], (float)rgb[1], (float)rgb[2]};
        gamut(p, f);
        if (!isfinite(f[0]) || !isfinite(f[1]) || !isfinite(f[2])) return 0;
        for (int c = 0; c < 3; ++c) rgb[c] = f[c];
    }
    return 1;
}

/* :152 apply_output_encoding_device: linear output RGB -> encoded, clamped */
static void encode_lin(const Pack* p, double* rgb) {
    double lin[3];
    if (p->enc_iso) memcpy(lin, rgb, sizeof(lin));
    else mat3d(p->dwg, rgb, lin);
    for (int c = 0; c < 3; ++c) rgb[c] = p->enc_cctf ? (double)enc(p, (float)lin[c]) : lin[c];
    for (int c = 0; c < 3; ++c) rgb[c] = clamp01(rgb[c]);
}

/* :1700-1858: density -> encoded RGB; returns 0 on a scan failure */
static int scan_out(const Pack* p, const float* D, double* rgb) {
    if (!scan_lin(p, D, rgb, -1.0f)) return 0;
    encode_lin(p, rgb);
    return 1;
}

/* ---------------- packing (JuicerCudaFilmPayloads.cpp:28-197, JuicerCudaResources.cpp) ---------------- */

typedef struct {
    Pack p;
    float* lut_store;
} Packed;

/* 1 while the density planes handed to the render entry points already hold print
 * density (after the enlarger diffusion): the scan then runs without the print step.
 * Set by oracle_set_print_done; the oracle's Python wrappers reset it after the call. */
static int g_print_done = 0;
void oracle_set_print_done(int v) { g_print_done = v; }

static int pack(const FjPreparedHostData* h, Packed* out) {
    memset(out, 0, sizeof(*out));
    Pack* p = &out->p;
    const FjFilmExposure* ex = &h->film_exposure;
    p->method = (int)ex->method;
    p->input_cs = (int)ex->input_color_space;
    p->decode = (ex->flags & FJ_FILM_DECODE_CCTF) != 0;
    p->adapt = (ex->flags & FJ_FILM_ADAPT_INPUT) != 0;
    memcpy(p->m_rgb_xyz, ex->input_rgb_to_xyz, 36);
    memcpy(p->m_adapt, ex->input_xyz_adapt, 36);
    memcpy(p->m_xyz_srgb, ex->xyz_to_linear_srgb, 36);
    p->tc = ex->tc_lut_rgba.data;
    p->mallett_basis = ex->mallett_basis.data;
    p->mallett_illum = ex->mallett_illuminant.data;
    for (int i = 0; i < NL; ++i)
        for (int bgr = 0; bgr < 3; ++bgr) p->sens_bgr[bgr][i] = ex->sensitivity_rgb.data[i * 3 + (2 - bgr)];
    p->mallett_midgray = ex->mallett_green_midgray_scale;
    p->manual = exp2f(ex->manual_exposure_ev);
    p->route = ex->route_correction_scale;
    const FjFilmDevelopment* dv = &h->film_development;
    const int n = (int)dv->log_exposure.count;
    for (int bgr = 0; bgr < 3; ++bgr) {
        int rgb = 2 - bgr;
        p->gamma_bgr[bgr] = dv->gamma_rgb[rgb];
        p->dens[bgr] = (Curve){dv->log_exposure.data, dv->density_rgb.data + rgb, 3, n};
    }
    const FjDirCouplers* dir = &h->dir_couplers;
    p->dir_mode = (int)dir->mode;
    if (dir->mode != FJ_DIR_INACTIVE) {
        for (int d = 0; d < 3; ++d) {
            for (int r = 0; r < 3; ++r) p->M[d * 3 + r] = dir->matrix_rgb[(2 - d) * 3 + (2 - r)];
            p->dmax[d] = dir->density_max_rgb[2 - d];
            p->dref[d] = dir->density_ref_rgb[2 - d];
            p->dk[d] = dir->donor_k_rgb[2 - d];
            p->rcref[d] = dir->receiver_c_ref_rgb[2 - d];
            p->rkr[d] = dir->receiver_kr_rgb[2 - d];
            p->dirc[d] = (Curve){dir->compensated_axes_rgb[2 - d].data, dv->density_rgb.data + (2 - d), 3, n};
        }
    }
    p->print = (h->route == FJ_ROUTE_NEGATIVE_PRINT || h->route == FJ_ROUTE_POSITIVE_PRINT) && !g_print_done;
    if (p->print) {
        const FjPrint* pr = &h->print;
        p->eps_c_src = pr->film_density_cmy.data;
        p->base_src = pr->film_base_density.data;
        p->pillum = pr->main_illuminant.data;
        p->psens = pr->sensitivity_cmy.data;
        p->print_exposure = pr->exposure;
        p->print_route = h->scanner_correction.exposure_scale;
        int pf = (pr->flags & FJ_PRINT_PREFLASH) != 0;
        p->preflash = pf ? pr->preflash_exposure : 0.0f;
        for (int c = 0; c < 3; ++c) p->preflash_raw[c] = pf ? pr->preflash_raw_cmy[c] : 0.0f;
        p->midgray = pr->normalizer;
        int np = (int)pr->log_exposure.count;
        for (int c = 0; c < 3; ++c) p->pdc[c] = (Curve){pr->log_exposure.data, pr->density_cmy.data + c, 3, np};
    }
    p->medium_negative = p->print ? 0 : 1;
    for (int c = 0; c < 3; ++c) {
        p->min_cmy[c] = p->print ? h->scanner_bounds.min_cmy[c] : -h->scanner_bounds.min_cmy[c];
        p->inv_cmy[c] = h->scanner_bounds.inv_span_cmy[c];
    }
    /* scanner LUT built on the host in FP64 */
    const FjScannerSpectra* sp = &h->scanner_spectra;
    int r = (int)h->scanner_lut.resolution;
    size_t nodes = (size_t)r * r * r * 3, cells = (size_t)(r - 1) * (r - 1) * (r - 1) * 3;
    out->lut_store = (float*)malloc((nodes * 4 + cells * 2) * sizeof(float));
    if (!out->lut_store) return 1;
    p->lut_v = out->lut_store;
    p->lut_sc = p->lut_v + nodes;
    p->lut_sm = p->lut_sc + nodes;
    p->lut_sy = p->lut_sm + nodes;
    p->cell_lo = p->lut_sy + nodes;
    p->cell_hi = p->cell_lo + cells;
    FjbScannerLutInput in;
    memset(&in, 0, sizeof(in));
    in.eps_c = sp->dye_c;
    in.eps_m = sp->dye_m;
    in.eps_y = sp->dye_y;
    in.weighted_x = sp->weighted_x;
    in.weighted_y = sp->weighted_y;
    in.weighted_z = sp->weighted_z;
    in.baseline_min = sp->base_density;
    in.has_baseline = sp->base_density.count != 0;
    in.sample_count = (int32_t)sp->dye_c.count;
    in.inv_yn = sp->inverse_y_normalization;
    for (int c = 0; c < 3; ++c) {
        in.range_min_cmy[c] = p->min_cmy[c];
        in.inverse_span_cmy[c] = p->inv_cmy[c];
    }
    in.medium = p->print ? 1u : 0u;
    in.resolution = (uint32_t)r;
    if (oracle_scanner_lut(&in, p->lut_v, p->lut_sc, p->lut_sm, p->lut_sy, p->cell_lo, p->cell_hi) != 0) return 2;
    p->res = r;
    p->corr_active = (h->scanner_correction.flags & FJ_CORRECTION_ACTIVE) != 0;
    p->corr_slope = h->scanner_correction.xyz_slope;
    p->corr_offset = h->scanner_correction.xyz_offset;
    const FjOutputColor* oc = &h->output_color;
    memcpy(p->cat02, oc->cat02, 36);
    memcpy(p->illum_xyz, oc->illuminant_xyz, 12);
    memcpy(p->xyz_rgb, oc->xyz_to_rgb, 36);
    p->gamut = (oc->flags & FJ_COLOR_GAMUT_COMPRESSION) != 0;
    p->cmax = oc->gamut_cmax.data;
    memcpy(p->g_to_xyz, oc->native_rgb_to_d65_xyz, 36);
    memcpy(p->g_from_xyz, oc->d65_xyz_to_native_rgb, 36);
    memcpy(p->lknee, oc->lightness_knee, 12);
    memcpy(p->cknee, oc->chroma_knee, 12);
    p->enc_iso = (oc->flags & FJ_COLOR_INPUT_IS_OUTPUT_SPACE) != 0;
    p->enc_cctf = (oc->flags & FJ_COLOR_ENCODE_CCTF) != 0;
    memcpy(p->dwg, oc->encoding.dwg_to_output, 36);
    p->cctf_kind = (int)oc->encoding.cctf_kind;
    p->cg = oc->encoding.gamma;
    p->ca = oc->encoding.a;
    p->cb = oc->encoding.b;
    p->cc = oc->encoding.c;
    p->cd = oc->encoding.d;
    p->ccut = oc->encoding.linear_cutoff;
    return 0;
}

/* ---------------- entry points ---------------- */

/* Stage selector: 0 = source -> encoded output; 1 = source -> capture density planes;
 * 2 = density planes -> encoded output; 3 = source -> camera exposure planes (B,G,R, no
 * route correction); 4 = carrier planes -> encoded output; 5 = carrier planes -> capture
 * density planes; 6 = source -> camera exposure planes with the route correction (the
 * film exposure the capture development takes); 7 = source -> the scanner's linear
 * output RGB planes R, G, B (before output gamut compression and encoding; NaN where the
 * scan fails). */
int oracle_render(const FjPreparedHostData* h, int stage, const float* src, long src_row_floats, int width,
                  int height, int comps, float* dst, long dst_row_floats, float* p0, float* p1, float* p2,
                  float auto_scale, int threads, unsigned* flags_out) {
    Packed pk;
    int rc = pack(h, &pk);
    if (rc) {
        free(pk.lut_store);
        return rc;
    }
    const Pack* p = &pk.p;
    Pack linear_pack = pk.p; /* stage 7: the scan without output gamut compression */
    linear_pack.gamut = 0;
    unsigned flags = 0;
#if defined(_OPENMP)
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads > 0 ? threads : 1) reduction(| : flags)
#endif
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < width; ++x) {
            size_t i = (size_t)y * width + x;
            const float* s = src ? src + (size_t)y * src_row_floats + (size_t)x * comps : NULL;
            float D[3];
            if (stage == 2) {
                D[0] = p0[i];
                D[1] = p1[i];
                D[2] = p2[i];
            } else if (stage == 4 || stage == 5) {
                float e[3] = {p0[i], p1[i], p2[i]};
                for (int c = 0; c < 3; ++c) e[c] = fmaxf(0.0f, e[c] * p->route);
                unsigned f = capture_density(p, e, D);
                if (f) flags |= (1u << 8) | ((f & 7u) << 9);
                if (stage == 5) { /* carrier B, G, R -> density C, M, Y in the same planes */
                    p0[i] = D[0];
                    p1[i] = D[1];
                    p2[i] = D[2];
                    continue;
                }
            } else {
                float e[3];
                film_exposure(p, s, auto_scale, stage == 3 ? 0 : 1, e);
                if (stage == 3 || stage == 6) {
                    p0[i] = e[0];
                    p1[i] = e[1];
                    p2[i] = e[2];
                    continue;
                }
                unsigned f = capture_density(p, e, D);
                if (f) flags |= (1u << 8) | ((f & 7u) << 9);
            }
            if (stage == 1) {
                p0[i] = D[0];
                p1[i] = D[1];
                p2[i] = D[2];
                continue;
            }
            if (p->print) print_stage(p, D);
            if (stage == 7) {
                double lin[3];
                const int ok = scan_lin(&linear_pack, D, lin, -1.0f);
                if (!ok) flags |= 1u;
                p0[i] = ok ? (float)lin[0] : nanf("");
                p1[i] = ok ? (float)lin[1] : nanf("");
                p2[i] = ok ? (float)lin[2] : nanf("");
                continue;
            }
            double rgb[3];
            float* o = dst + (size_t)y * dst_row_floats + (size_t)x * comps;
            if (!scan_out(p, D, rgb)) {
                flags |= 1u;
                o[0] = o[1] = o[2] = 0.0f;
            } else {
                o[0] = (float)rgb[0];
                o[1] = (float)rgb[1];
                o[2] = (float)rgb[2];
            }
            if (comps == 4) o[3] = s ? s[3] : 1.0f;
        }
    }
    free(pk.lut_store);
    if (flags_out) *flags_out = flags;
    return 0;
}

/* ---------------- auto exposure (src/Cuda/JuicerCudaAutoExposure.cu:63-141, :266-520) ---------------- */

static int preview_coord(int i, int preview, int source) {
    if (preview <= 0 || source <= 0) return 0;
    long long num = (2LL * i + 1LL) * (long long)source;
    int c = (int)(num / (2LL * preview));
    return c < 0 ? 0 : (c > source - 1 ? source - 1 : c);
}

static void meter_w(int method, int x, int y, int w, int h, float lum, float* out) {
    for (int l = 0; l < 4; ++l) out[l] = 0.0f;
    if (method == FJ_METER_AVERAGE || method == FJ_METER_MEDIAN) {
        out[0] = 1.0f;
        return;
    }
    int maxDim = w > h ? w : h;
    float invMax = maxDim > 0 ? 1.0f / (float)maxDim : 0.0f;
    if (method == FJ_METER_CENTER_WEIGHTED) {
        const float sg = 0.2f;
        float nx = ((float)x / (float)w) - 0.5f, normX = nx * (float)w * invMax;
        float ny = ((float)y / (float)h) - 0.5f, normY = ny * (float)h * invMax;
        out[0] = expf(-(normX * normX) / (2.0f * sg * sg)) * expf(-(normY * normY) / (2.0f * sg * sg));
        return;
    }
    float nx = (((float)x / (float)w) - 0.5f) * (float)w * invMax;
    float ny = (((float)y / (float)h) - 0.5f) * (float)h * invMax;
    float radius = sqrtf(nx * nx + ny * ny);
    if (method == FJ_METER_PARTIAL) {
        out[0] = radius < 0.15f ? 1.0f : 0.0f;
        out[3] = 1.0f;
    } else if (method == FJ_METER_MATRIX) {
        int ch = h / 5, cw = w / 5;
        if (ch <= 0 || cw <= 0) return;
        int row = y / ch, col = x / cw;
        if (row >= 5 || col >= 5) return;
        float dy = ((float)row - 2.0f) / 2.0f, dx = ((float)col - 2.0f) / 2.0f;
        float dist = sqrtf(dx * dx + dy * dy) / sqrtf(2.0f);
        out[0] = 0.5f * (1.0f + cosf(3.14159265358979323846f * dist));
    } else if (method == FJ_METER_MULTI_ZONE) {
        if (radius >= 0.0f && radius < 0.05f) out[0] = 1.0f;
        else if (radius >= 0.05f && radius < 0.25f) out[1] = 1.0f;
        else if (radius >= 0.25f && radius < 0.50f) out[2] = 1.0f;
        out[3] = 1.0f;
    } else if (method == FJ_METER_HIGHLIGHT_WEIGHTED) {
        out[0] = lum * lum;
        out[3] = 1.0f;
    }
}

/* Returns the exposure scale; *ok = 0 for rejected records (median, empty windows). */
float oracle_auto_exposure(const FjPreparedHostData* h, const FjAutoExposure* m, const float* src, long src_row_floats,
                           int comps, int* ok) {
    *ok = 0;
    if (m->method == FJ_METER_MEDIAN || m->preview_width <= 0 || m->preview_height <= 0) return 1.0f;
    Packed pk;
    if (pack(h, &pk)) {
        free(pk.lut_store);
        return 1.0f;
    }
    const Pack* p = &pk.p;
    double Y[4] = {0, 0, 0, 0}, W[4] = {0, 0, 0, 0};
    int pw = m->preview_width, ph = m->preview_height;
    int sw = m->meter_bounds.x2 - m->meter_bounds.x1, sh = m->meter_bounds.y2 - m->meter_bounds.y1;
    for (int y = 0; y < ph; ++y) {
        int py = m->meter_bounds.y1 + preview_coord(y, ph, sh);
        if (py < m->source_bounds.y1 || py >= m->source_bounds.y2) continue;
        for (int x = 0; x < pw; ++x) {
            int px = m->meter_bounds.x1 + preview_coord(x, pw, sw);
            if (px < m->source_bounds.x1 || px >= m->source_bounds.x2) continue;
            const float* s = src + (size_t)(py - m->source_bounds.y1) * src_row_floats +
                             (size_t)(px - m->source_bounds.x1) * comps;
            float raw[3];
            if (p->method == FJ_RAW_MALLETT_2019) mallett_exposure(p, s, raw);
            else tc_exposure(p, s, raw);
            float mean = (raw[0] + raw[1] + raw[2]) * (1.0f / 3.0f);
            if (!isfinite(mean)) continue;
            float w[4];
            meter_w((int)m->method, x, y, pw, ph, mean, w);
            for (int l = 0; l < 4; ++l) {
                float wl = (isfinite(w[l]) && w[l] > 0.0f) ? w[l] : 0.0f;
                Y[l] += (double)mean * (double)wl;
                W[l] += (double)wl;
            }
        }
    }
    free(pk.lut_store);
    double yexp = 0.0;
    int has = 0;
    if (m->method == FJ_METER_PARTIAL) {
        int l = W[0] > 0.0 ? 0 : 3;
        if (W[l] > 0.0) {
            yexp = Y[l] / W[l];
            has = 1;
        }
    } else if (m->method == FJ_METER_MULTI_ZONE) {
        const double ring[3] = {0.50, 0.30, 0.20};
        double ws = 0.0, wt = 0.0;
        for (int l = 0; l < 3; ++l)
            if (W[l] > 0.0) {
                ws += ring[l] * Y[l] / W[l];
                wt += ring[l];
            }
        if (wt > 0.0) {
            yexp = ws / wt;
            has = 1;
        } else if (W[3] > 0.0) {
            yexp = Y[3] / W[3];
            has = 1;
        }
    } else if (m->method == FJ_METER_HIGHLIGHT_WEIGHTED && W[0] < 1e-12) {
        if (W[3] > 0.0) {
            yexp = Y[3] / W[3];
            has = 1;
        }
    } else if (W[0] > 0.0) {
        yexp = Y[0] / W[0];
        has = 1;
    }
    double ev = 0.0;
    if (has && isfinite(yexp) && yexp > 0.0) {
        double c = -log(yexp / 1.0) / log(2.0);
        if (isfinite(c)) ev = c;
    }
    double s64 = exp2(ev);
    *ok = 1;
    return (isfinite(s64) && s64 > 0.0) ? (float)s64 : 1.0f;
}

/* ---------------- scatter / halation (src/Cuda/Film/JuicerCudaScatterHalation.cu) ----------------
 * Literal per-channel schedule of launch_scatter_halation (:690-852): accumulation
 * buffer cleared, each tail Gaussian accumulated with its amplitude, the core pass
 * combined with the source, then the bounces accumulated and added. FIR Gaussians
 * filter columns first then rows (:483-526); YVV Gaussians rows first (forward then
 * backward) then columns (bottom-up then top-down) (:201-345). */

static int reflect_half(int i, int n) {
    if (i >= 0 && i < n) return i;
    if (i >= -n && i < 0) return -i - 1;
    if (i >= n && i < 2 * n) return 2 * n - 1 - i;
    int period = 2 * n;
    i %= period;
    if (i < 0) i += period;
    return i >= n ? period - 1 - i : i;
}

typedef struct {
    float s1, s2, s3;
} Yvv;

static void yvv_init(const FjHalationGaussian* g, float first, Yvv* s) {
    s->s1 = first;
    s->s2 = first;
    s->s3 = g->kind == FJ_HALATION_YVV_REPLICATE_FACTORED ? 0.0f : first;
}

static float yvv_step(const FjHalationGaussian* g, float x, Yvv* s) {
    if (g->kind == FJ_HALATION_YVV_REPLICATE_FACTORED) {
        s->s1 += g->yvv[0] * (x - s->s1);
        s->s3 = g->yvv[2] * s->s3 + g->yvv[1] * (s->s1 - s->s2);
        s->s2 += s->s3;
        return s->s2;
    }
    float v = g->yvv[0] * x + g->yvv[1] * s->s1 + g->yvv[2] * s->s2 + g->yvv[3] * s->s3;
    s->s3 = s->s2;
    s->s2 = s->s1;
    s->s1 = v;
    return v;
}

/* Gaussian of `src` (stride sstride) into `out` (width stride); tmp is scratch. */
static void gauss(const FjHalationGaussian* g, const float* src, long sstride, float* out, float* tmp, int W, int H) {
    if (g->kind == FJ_HALATION_IDENTITY) {
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) out[(size_t)y * W + x] = src[(size_t)y * sstride + x];
        return;
    }
    if (g->kind == FJ_HALATION_FIR_REFLECT) {
        int r = g->radius;
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                float s = 0.0f;
                for (int o = -r; o <= r; ++o) s += src[(size_t)reflect_half(y - o, H) * sstride + x] * g->fir_weights[o + r];
                tmp[(size_t)y * W + x] = s;
            }
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                float s = 0.0f;
                for (int o = -r; o <= r; ++o) s += tmp[(size_t)y * W + reflect_half(x + o, W)] * g->fir_weights[o + r];
                out[(size_t)y * W + x] = s;
            }
        return;
    }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        Yvv s;
        yvv_init(g, src[(size_t)y * sstride], &s);
        for (int x = 0; x < W; ++x) tmp[(size_t)y * W + x] = yvv_step(g, src[(size_t)y * sstride + x], &s);
        yvv_init(g, tmp[(size_t)y * W + W - 1], &s);
        for (int x = W - 1; x >= 0; --x) tmp[(size_t)y * W + x] = yvv_step(g, tmp[(size_t)y * W + x], &s);
    }
#pragma omp parallel for schedule(static)
    for (int x = 0; x < W; ++x) {
        Yvv s;
        yvv_init(g, tmp[(size_t)(H - 1) * W + x], &s);
        for (int y = H - 1; y >= 0; --y) tmp[(size_t)y * W + x] = yvv_step(g, tmp[(size_t)y * W + x], &s);
        yvv_init(g, tmp[x], &s);
        for (int y = 0; y < H; ++y) out[(size_t)y * W + x] = yvv_step(g, tmp[(size_t)y * W + x], &s);
    }
}

/* planes: R, G, B planes of width W, row stride `stride` floats, modified in place. */
int oracle_scatter_halation(const FjScatterHalation* d, float* r, float* g, float* b, long stride, int W, int H) {
    static const float amp[3] = {0.1633f, 0.6496f, 0.1870f};
    size_t n = (size_t)W * H;
    float* acc = (float*)calloc(n, sizeof(float));
    float* val = (float*)malloc(n * sizeof(float));
    float* tmp = (float*)malloc(n * sizeof(float));
    float* planes[3] = {r, g, b};
    if (!acc || !val || !tmp) return 1;
    for (int c = 0; c < 3; ++c) {
        float* P = planes[c];
        const FjHalationChannel* ch = &d->channels[c];
        if (d->scatter_amount != 0.0f) {
            int tails = ch->tail_weight > 0.0f;
            if (tails) {
                for (int i = 0; i < 3; ++i) {
                    gauss(&ch->tail[i], P, stride, val, tmp, W, H);
                    for (size_t k = 0; k < n; ++k) acc[k] = i == 0 ? amp[i] * val[k] : acc[k] + amp[i] * val[k];
                }
            }
            gauss(&ch->core, P, stride, val, tmp, W, H);
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    size_t k = (size_t)y * W + x;
                    float source = P[(size_t)y * stride + x];
                    float tail = tails ? acc[k] : 0.0f;
                    float coreTerm = (1.0f - ch->tail_weight) * val[k];
                    float tailTerm = ch->tail_weight * tail;
                    float scattered = coreTerm + tailTerm;
                    float sourceTerm = (1.0f - d->scatter_amount) * source;
                    float scatteredTerm = d->scatter_amount * scattered;
                    P[(size_t)y * stride + x] = sourceTerm + scatteredTerm;
                }
        }
        if (ch->total_strength == 0.0f) continue;
        memset(acc, 0, n * sizeof(float));
        for (unsigned i = 0; i < d->bounce_count; ++i) {
            gauss(&ch->bounce[i], P, stride, val, tmp, W, H);
            for (size_t k = 0; k < n; ++k) acc[k] = i == 0 ? d->bounce_weights[i] * val[k] : acc[k] + d->bounce_weights[i] * val[k];
        }
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                float source = P[(size_t)y * stride + x];
                float added = source + ch->total_strength * acc[(size_t)y * W + x];
                P[(size_t)y * stride + x] = d->renormalize ? added / (1.0f + ch->total_strength) : added;
            }
    }
    free(acc);
    free(val);
    free(tmp);
    return 0;
}

/* ---------------- spatial DIR boundaries (rust/film-juicer-core/src/film/dir/boundary.rs:207-503) ----------------
 *
 * The reflected Young-van Vliet start weights and end matrix of one axis, in the
 * reference's double-double arithmetic (a value is the unevaluated sum hi + lo; sums
 * are Knuth two-sums folded into a fast renormalisation, products carry the exact
 * residual fma(a, b, -a*b)). The operation order follows boundary.rs step by step so
 * that the binary64 results are the reference's words. */

typedef struct {
    double h, l;
} DDv;

static DDv ddv(double v) {
    DDv r = {v, 0.0};
    return r;
}
static DDv dd_renorm(double h, double l) { /* boundary.rs:215-221 */
    DDv r;
    r.h = h + l;
    r.l = l - (r.h - h);
    return r;
}
static DDv dd_plus(DDv a, DDv b) { /* :222-227 */
    double s = a.h + b.h;
    double v = s - a.h;
    return dd_renorm(s, (a.h - (s - v)) + (b.h - v) + a.l + b.l);
}
static DDv dd_minus(DDv a, DDv b) {
    DDv nb = {-b.h, -b.l};
    return dd_plus(a, nb);
}
static DDv dd_times(DDv a, DDv b) { /* :237-245 */
    double p = a.h * b.h;
    return dd_renorm(p, fma(a.h, b.h, -p) + a.h * b.l + a.l * b.h + a.l * b.l);
}
static DDv dd_over(DDv a, DDv d) { /* :246-251 */
    double q1 = a.h / d.h;
    DDv rem = dd_minus(a, dd_times(d, ddv(q1)));
    double q2 = (rem.h + rem.l) / d.h;
    return dd_plus(ddv(q1), ddv(q2));
}
static double dd_val(DDv a) { return a.h + a.l; }

/* o = m v for a 3x3 matrix (row-major) and a 3-vector (:276-284) */
static void dd_matvec(const DDv* m, const DDv* v, DDv* o) {
    DDv t[3];
    for (int r = 0; r < 3; ++r) {
        t[r] = ddv(0.0);
        for (int c = 0; c < 3; ++c) t[r] = dd_plus(t[r], dd_times(m[r * 3 + c], v[c]));
    }
    memcpy(o, t, sizeof t);
}

/* o = a b (:264-274) */
static void dd_matmul(const DDv* a, const DDv* b, DDv* o) {
    DDv t[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            t[r * 3 + c] = ddv(0.0);
            for (int k = 0; k < 3; ++k) t[r * 3 + c] = dd_plus(t[r * 3 + c], dd_times(a[r * 3 + k], b[k * 3 + c]));
        }
    memcpy(o, t, sizeof t);
}

static void dd_eye(DDv* m) {
    for (int i = 0; i < 9; ++i) m[i] = ddv(i % 4 == 0 ? 1.0 : 0.0);
}

/* Gauss-Jordan inverse of the leading n x n block with partial pivoting on the
 * rounded magnitudes (:286-320). Returns 0 when a pivot is zero or not finite. */
static int dd_inverse(DDv* m, int n, DDv* inv) {
    dd_eye(inv);
    for (int col = 0; col < n; ++col) {
        int piv = col;
        double best = fabs(dd_val(m[col * 3 + col]));
        for (int r = col + 1; r < n; ++r)
            if (fabs(dd_val(m[r * 3 + col])) > best) {
                best = fabs(dd_val(m[r * 3 + col]));
                piv = r;
            }
        if (!(best > 0.0 && isfinite(best))) return 0;
        if (piv != col)
            for (int j = 0; j < 3; ++j) {
                DDv t = m[piv * 3 + j];
                m[piv * 3 + j] = m[col * 3 + j];
                m[col * 3 + j] = t;
                t = inv[piv * 3 + j];
                inv[piv * 3 + j] = inv[col * 3 + j];
                inv[col * 3 + j] = t;
            }
        DDv s = m[col * 3 + col];
        for (int j = 0; j < n; ++j) {
            m[col * 3 + j] = dd_over(m[col * 3 + j], s);
            inv[col * 3 + j] = dd_over(inv[col * 3 + j], s);
        }
        for (int r = 0; r < n; ++r) {
            if (r == col) continue;
            DDv f = m[r * 3 + col];
            for (int j = 0; j < n; ++j) {
                m[r * 3 + j] = dd_minus(m[r * 3 + j], dd_times(f, m[col * 3 + j]));
                inv[r * 3 + j] = dd_minus(inv[r * 3 + j], dd_times(f, inv[col * 3 + j]));
            }
        }
    }
    return 1;
}

static long long reflect_ll(long long i, long long n) { /* boundary.rs:491-502 */
    long long p = 2 * n, w = i % p;
    if (w < 0) w += p;
    return w < n ? w : p - 1 - w;
}

/* One axis of the boundary (boundary.rs:361-489). coeff: normalised feedforward,
 * feedback[3], unnormalised denominator, feedforward numerator, feedback
 * numerators[3]. weights receives 3 x retained start weights (row-major by state
 * row; capacity 3 L), terminal the ts x ts end matrix. Returns 0, or the reference's
 * Reason code: 4 policy, 5 causal singular, 6 non-finite weights, 7 causal
 * certification, 8 tail escape, 9 terminal singular, 10 terminal certification,
 * 12 allocation. */
int oracle_dir_boundary(const double* coeff, double accuracy, double tolerance, unsigned version, int L,
                        double* weights, int* retained_out, int* ts_out, double* terminal) {
    if (L <= 0 || !(accuracy > 0.0 && tolerance > 0.0) || version != 1) return 4;
    const long long period = 2LL * L;
    DDv A[9];
    for (int i = 0; i < 9; ++i) A[i] = ddv(0.0);
    A[0] = ddv(coeff[1]);
    A[1] = ddv(coeff[2]);
    A[2] = ddv(coeff[3]);
    A[3] = ddv(1.0);
    A[7] = ddv(1.0);
    /* impulse responses b, A b, A^2 b, ... with b = (ff, 0, 0) */
    DDv* pw = (DDv*)malloc((size_t)period * 3 * sizeof(DDv));
    double* full = (double*)malloc((size_t)L * 3 * sizeof(double));
    if (!pw || !full) {
        free(pw);
        free(full);
        return 12;
    }
    pw[0] = ddv(coeff[0]);
    pw[1] = pw[2] = ddv(0.0);
    for (long long e = 1; e < period; ++e) dd_matvec(A, pw + (e - 1) * 3, pw + e * 3);
    /* I - A^(2L), A^(2L) accumulated as A (A (... I)) */
    DDv P[9], S[9], Si[9];
    dd_eye(P);
    for (long long e = 0; e < period; ++e) dd_matmul(A, P, P);
    dd_eye(S);
    for (int i = 0; i < 9; ++i) S[i] = dd_minus(S[i], P[i]);
    int rc = 0;
    if (!dd_inverse(S, 3, Si)) rc = 5;
    DDv sums[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int s = 0; !rc && s < L; ++s) {
        DDv rhs[3], st[3];
        for (int r = 0; r < 3; ++r) rhs[r] = dd_plus(pw[s * 3 + r], pw[(period - 1 - s) * 3 + r]);
        dd_matvec(Si, rhs, st);
        for (int r = 0; r < 3; ++r) {
            double v = dd_val(st[r]);
            if (!isfinite(v)) {
                rc = 6;
                break;
            }
            full[(size_t)r * L + s] = v;
            sums[r] = dd_plus(sums[r], ddv(v));
        }
    }
    for (int r = 0; !rc && r < 3; ++r) {
        double v = dd_val(sums[r]);
        if (!isfinite(v) || fabs(v - 1.0) > tolerance) rc = 7;
    }
    free(pw);
    if (rc) {
        free(full);
        return rc;
    }
    /* truncation: drop trailing samples while the tail mass of every row stays below
     * the accuracy (never below min(L, 3) samples) */
    int lo = L < 3 ? L : 3, keep = L;
    double tail[3] = {0.0, 0.0, 0.0};
    for (int s = L - 1; s >= lo; --s) {
        for (int r = 0; r < 3; ++r) tail[r] += fabs(full[(size_t)r * L + s]);
        if (fmax(fmax(tail[0], tail[1]), tail[2]) >= accuracy) {
            keep = s + 1;
            break;
        }
        keep = s;
    }
    for (int r = 0; r < 3; ++r)
        for (int s = 0; s < keep; ++s) weights[(size_t)r * keep + s] = full[(size_t)r * L + s];
    free(full);
    /* end block: denominator on the diagonal minus the reflected feedback numerators */
    const int n = L < 3 ? L : 3;
    DDv T[9], Ti[9];
    for (int i = 0; i < 9; ++i) T[i] = ddv(0.0);
    for (int d = 0; d < n; ++d) T[d * 3 + d] = ddv(coeff[4]);
    for (int row = 0; row < n; ++row)
        for (int k = 0; k < 3; ++k) {
            long long col = reflect_ll((long long)(L - n + row) + k + 1, L) - (L - n);
            if (col < 0 || col >= n) return 8;
            T[row * 3 + col] = dd_minus(T[row * 3 + col], ddv(coeff[6 + k]));
        }
    if (!dd_inverse(T, n, Ti)) return 9;
    for (int i = 0; i < 9; ++i) terminal[i] = 0.0;
    for (int row = 0; row < n; ++row) {
        double sum = 0.0;
        for (int c = 0; c < n; ++c) {
            double v = dd_val(dd_times(ddv(coeff[5]), Ti[row * 3 + c]));
            terminal[row * n + c] = v;
            sum += v;
        }
        if (!isfinite(sum) || fabs(sum - 1.0) > tolerance) return 10;
    }
    *retained_out = keep;
    *ts_out = n;
    return 0;
}

/* ---------------- spatial DIR (src/Cuda/Film/JuicerCudaFilmPipeline.cu:124-1060) ---------------- */

typedef struct {
    int op; /* 1 identity, 2 FIR, 3 recursive */
    float weight;
    int radius;
    const float* taps;
    double ff, fb[3];
    const double* h_init;
    int h_len, h_ts;
    double h_term[9];
    const double* v_init;
    int v_len, v_ts;
    double v_term[9];
} OracleDirComp;

static int reflect_dir(int i, int n) {
    if (n <= 1) return 0;
    int period = 2 * n;
    i %= period;
    if (i < 0) i += period;
    return i >= n ? period - 1 - i : i;
}

static double iir(const OracleDirComp* c, double x, double* s) {
    double v = c->ff * x + c->fb[0] * s[0] + c->fb[1] * s[1] + c->fb[2] * s[2];
    s[2] = s[1];
    s[1] = s[0];
    s[0] = v;
    return v;
}

/* Raw donor corrections (Y, M, C) and raw log exposure (B, G, R) per pixel, from the
 * source image (carrier == NULL) or carrier planes B, G, R (:124-214). */
int oracle_dir_source(const FjPreparedHostData* h, const float* src, long src_row_floats, int comps,
                      const float* cb, const float* cg, const float* cr, int W, int H, float* y_out, float* m_out,
                      float* c_out, float* lb, float* lg, float* lr, unsigned* flags_out) {
    Packed pk;
    if (pack(h, &pk)) {
        free(pk.lut_store);
        return 1;
    }
    const Pack* p = &pk.p;
    unsigned flags = 0;
#pragma omp parallel for schedule(static) reduction(| : flags)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t i = (size_t)y * W + x;
            float e[3];
            if (cb) {
                e[0] = fmaxf(0.0f, cb[i] * p->route);
                e[1] = fmaxf(0.0f, cg[i] * p->route);
                e[2] = fmaxf(0.0f, cr[i] * p->route);
            } else {
                film_exposure(p, src + (size_t)y * src_row_floats + (size_t)x * comps, 1.0f, 1, e);
            }
            float logE[3], layer[3];
            for (int c = 0; c < 3; ++c) {
                logE[c] = log10f(fmaxf(e[c], 0.0f) + 1e-10f);
                layer[c] = curve_at(&p->dens[c], inf_clamp(&p->dens[c], logE[c]), p->gamma_bgr[c]);
            }
            float donor[3] = {p->dmax[0] - layer[0], p->dmax[1] - layer[1], p->dmax[2] - layer[2]};
            unsigned fail = 0;
            if (p->dir_mode == FJ_DIR_NEGATIVE_DONOR_LANGMUIR)
                for (int c = 0; c < 3; ++c)
                    if (!langmuir(layer[c], p->dk[c], p->dref[c], &donor[c])) fail |= 1u << c;
            float corr[3];
            corr[0] = p->M[0] * donor[0] + p->M[3] * donor[1] + p->M[6] * donor[2];
            corr[1] = p->M[1] * donor[0] + p->M[4] * donor[1] + p->M[7] * donor[2];
            corr[2] = p->M[2] * donor[0] + p->M[5] * donor[1] + p->M[8] * donor[2];
            for (int c = 0; c < 3; ++c)
                if (!isfinite(corr[c])) fail |= 1u << c;
            if (fail) flags |= (1u << 8) | ((fail & 7u) << 9);
            y_out[i] = corr[0];
            m_out[i] = corr[1];
            c_out[i] = corr[2];
            lb[i] = logE[0];
            lg[i] = logE[1];
            lr[i] = logE[2];
        }
    free(pk.lut_store);
    if (flags_out) *flags_out = flags;
    return 0;
}

/* filtered = sum over components in order of weight * G(raw), the reference's
 * per-component schedule (:940-1060) with its FP64 accumulations. */
int oracle_dir_blur(const OracleDirComp* comps, int n, const float* raw, int W, int H, float* filtered) {
    size_t N = (size_t)W * H;
    float* tmp = (float*)malloc(N * sizeof(float));
    float* fwd = (float*)malloc(N * sizeof(float));
    if (!tmp || !fwd) return 1;
    int first = 1;
    for (int k = 0; k < n; ++k) {
        const OracleDirComp* c = &comps[k];
        if (!(c->weight > 0.0f)) continue;
        if (c->op == 1) {
            for (size_t i = 0; i < N; ++i) {
                float wv = raw[i] * c->weight;
                filtered[i] = first ? wv : filtered[i] + wv;
            }
        } else if (c->op == 2) {
            int r = c->radius;
#pragma omp parallel for schedule(static)
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    double s = 0.0;
                    for (int o = -r; o <= r; ++o)
                        s += (double)raw[(size_t)y * W + reflect_dir(x + o, W)] * (double)c->taps[o + r];
                    tmp[(size_t)y * W + x] = isfinite(s) ? (float)s : 0.0f;
                }
#pragma omp parallel for schedule(static)
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    double s = 0.0;
                    for (int o = -r; o <= r; ++o)
                        s += (double)tmp[(size_t)reflect_dir(y + o, H) * W + x] * (double)c->taps[o + r];
                    float b = isfinite(s) ? (float)s : 0.0f;
                    float wv = b * c->weight;
                    size_t i = (size_t)y * W + x;
                    filtered[i] = first ? wv : filtered[i] + wv;
                }
        } else {
#pragma omp parallel for schedule(static)
            for (int y = 0; y < H; ++y) {
                const float* in = raw + (size_t)y * W;
                float* out = tmp + (size_t)y * W;
                double anchor = (double)in[0];
                double s[3] = {anchor, anchor, anchor};
                for (int i = 0; i < c->h_len; ++i) {
                    double d = (double)in[i] - anchor;
                    for (int hh = 0; hh < 3; ++hh) s[hh] += c->h_init[hh * c->h_len + i] * d;
                }
                for (int x = 0; x < W; ++x) out[x] = (float)iir(c, (double)in[x], s);
                int ts = c->h_ts;
                double term[3] = {0, 0, 0}, last = s[0];
                for (int rr = 0; rr < ts; ++rr) {
                    double v = last;
                    for (int q = 0; q < ts; ++q) v += c->h_term[rr * ts + q] * (s[ts - 1 - q] - last);
                    term[rr] = v;
                    out[W - ts + rr] = (float)v;
                }
                for (int hh = 0; hh < ts; ++hh) s[hh] = term[hh];
                for (int x = W - ts - 1; x >= 0; --x) out[x] = (float)iir(c, (double)out[x], s);
            }
#pragma omp parallel for schedule(static)
            for (int x = 0; x < W; ++x) {
                double anchor = (double)tmp[(size_t)(H - 1) * W + x];
                double s[3] = {anchor, anchor, anchor};
                for (int i = 0; i < c->v_len; ++i) {
                    double d = (double)tmp[(size_t)(H - 1 - i) * W + x] - anchor;
                    for (int hh = 0; hh < 3; ++hh) s[hh] += c->v_init[hh * c->v_len + i] * d;
                }
                for (int vy = 0; vy < H; ++vy) {
                    size_t i = (size_t)(H - 1 - vy) * W + x;
                    fwd[i] = (float)iir(c, (double)tmp[i], s);
                }
                int ts = c->v_ts;
                double term[3] = {0, 0, 0}, last = s[0];
                for (int rr = 0; rr < ts; ++rr) {
                    double v = last;
                    for (int q = 0; q < ts; ++q) v += c->v_term[rr * ts + q] * (s[ts - 1 - q] - last);
                    term[rr] = v;
                    int vy = H - ts + rr;
                    size_t i = (size_t)(H - 1 - vy) * W + x;
                    float wv = (float)v * c->weight;
                    filtered[i] = first ? wv : filtered[i] + wv;
                }
                for (int hh = 0; hh < ts; ++hh) s[hh] = term[hh];
                for (int vy = H - ts - 1; vy >= 0; --vy) {
                    size_t i = (size_t)(H - 1 - vy) * W + x;
                    double v = iir(c, (double)fwd[i], s);
                    float wv = (float)v * c->weight;
                    filtered[i] = first ? wv : filtered[i] + wv;
                }
            }
        }
        first = 0;
    }
    free(tmp);
    free(fwd);
    return 0;
}

/* Capture density from filtered corrections + cached log exposure
 * (src/Cuda/JuicerCudaDeviceHelpers.cuh:1267-1328); planes C, M, Y out. */
int oracle_develop_spatial(const FjPreparedHostData* h, const float* fy, const float* fm, const float* fc,
                           const float* lb, const float* lg, const float* lr, int W, int H, float* oc, float* om,
                           float* oy, unsigned* flags_out) {
    Packed pk;
    if (pack(h, &pk)) {
        free(pk.lut_store);
        return 1;
    }
    const Pack* p = &pk.p;
    unsigned flags = 0;
#pragma omp parallel for schedule(static) reduction(| : flags)
    for (long i = 0; i < (long)W * H; ++i) {
        float corr[3] = {fy[i], fm[i], fc[i]};
        unsigned fail = 0;
        if (p->dir_mode == FJ_DIR_POSITIVE_RECEIVER_LANGMUIR)
            for (int c = 0; c < 3; ++c) {
                if (p->rcref[c] == 0.0f) {
                    corr[c] = 0.0f;
                    continue;
                }
                float v = corr[c];
                if (!langmuir(v, p->rkr[c], p->rcref[c], &corr[c])) fail |= 1u << c;
            }
        float lc[3];
        const float lraw[3] = {lb[i], lg[i], lr[i]};
        if (!fail)
            for (int c = 0; c < 3; ++c) {
                float o = lraw[c];
                if (isnan(o)) {
                    fail |= 1u << c;
                    continue;
                }
                lc[c] = o - corr[c];
                if ((!isinf(o) && !isfinite(lc[c])) || (isinf(o) && (!isinf(lc[c]) || signbit(o) != signbit(lc[c]))))
                    fail |= 1u << c;
            }
        if (fail) {
            flags |= (1u << 8) | ((fail & 7u) << 9);
            oc[i] = om[i] = oy[i] = nanf("");
            continue;
        }
        for (int c = 0; c < 3; ++c) lc[c] = inf_clamp(&p->dens[c], lc[c]);
        oy[i] = curve_at(&p->dirc[0], lc[0], p->gamma_bgr[0]);
        om[i] = curve_at(&p->dirc[1], lc[1], p->gamma_bgr[1]);
        oc[i] = curve_at(&p->dirc[2], lc[2], p->gamma_bgr[2]);
    }
    free(pk.lut_store);
    if (flags_out) *flags_out = flags;
    return 0;
}

/* ---------------- diffusion (src/Cuda/Diffusion/JuicerCudaDiffusion.cu:294-487) ----------------
 * PSF in FP64, stored as float, normalised by the FP64 sum of the stored floats; the
 * convolution is evaluated directly in FP64 over the whole-sample-reflected frame
 * (the reference's reflect-padded FFT tiles compute the same linear convolution). */
static long reflect_whole(long i, long n) {
    if (n <= 1) return 0;
    long period = 2 * (n - 1);
    long v = i % period;
    if (v < 0) v += period;
    return v < n ? v : period - v;
}

/* The normalised (2r+1)^2 PSF of channel c (0 R, 1 G, 2 B) as stored floats. */
void oracle_diffusion_psf(const double* lambda_px, const double* weights, int radius, int c, float* psf) {
    int d = 2 * radius + 1;
    const double two_pi = 6.283185307179586476925286766559;
    double sum = 0.0;
    for (int iy = 0; iy < d; ++iy)
        for (int ix = 0; ix < d; ++ix) {
            int dx = ix - radius, dy = iy - radius;
            double rho = sqrt((double)dx * dx + (double)dy * dy);
            double v = 0.0;
            for (int k = 0; k < 9; ++k) {
                double l = lambda_px[k];
                v += weights[c * 9 + k] * exp(-rho / l) / (two_pi * l * l);
            }
            psf[(size_t)iy * d + ix] = (float)v;
            sum += (double)(float)v;
        }
    for (size_t i = 0; i < (size_t)d * d; ++i) psf[i] = (float)((double)psf[i] / sum);
}

int oracle_diffusion(const double* lambda_px, const double* weights /* [3][9] R,G,B */, int radius, double fraction,
                     const float* const* src, float* const* dst, int W, int H) {
    int d = 2 * radius + 1;
    float* psf = (float*)malloc((size_t)d * d * sizeof(float));
    if (!psf) return 1;
    for (int c = 0; c < 3; ++c) {
        oracle_diffusion_psf(lambda_px, weights, radius, c, psf);
        const float f = (float)fraction;
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                double acc = 0.0;
                for (int iy = 0; iy < d; ++iy) {
                    long sy = reflect_whole(y + iy - radius, H);
                    for (int ix = 0; ix < d; ++ix) {
                        long sx = reflect_whole(x + ix - radius, W);
                        acc += (double)psf[(size_t)iy * d + ix] * (double)src[c][sy * W + sx];
                    }
                }
                float cur = src[c][(size_t)y * W + x];
                dst[c][(size_t)y * W + x] = (1.0f - f) * cur + f * (float)acc;
            }
    }
    free(psf);
    return 0;
}

/* ---------------- enlarger diffusion (src/Cuda/Scan/JuicerCudaScanPipeline.cu:1392-1488) ----------------
 * Print-linear exposure of capture density planes: the spectral integral of the print
 * stage times the dust transmittance and the mid-grey normaliser, plus preflash, then
 * (max(raw, 0) + 1e-10) x print exposure x route correction
 * (src/Cuda/JuicerCudaDeviceHelpers.cuh:966-1010); planes C-, M-, Y-forming out. */
int oracle_enlarger_linear(const FjPreparedHostData* h, const float* dc, const float* dm, const float* dy,
                           const float* dust, int W, int H, float* lc, float* lm, float* ly) {
    Packed pk;
    if (pack(h, &pk) || !pk.p.print) {
        free(pk.lut_store);
        return 1;
    }
    const Pack* p = &pk.p;
    const float outer = p->print_exposure * p->print_route;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)W * H; ++i) {
        float D[3] = {dc[i], dm[i], dy[i]}, raw[3];
        print_spectral_raw(p, D, raw);
        float t = dust ? dust[i] : 1.0f;
        if (t != 1.0f)
            for (int c = 0; c < 3; ++c) raw[c] *= t;
        for (int c = 0; c < 3; ++c) raw[c] *= p->midgray;
        if (p->preflash > 0.0f)
            for (int c = 0; c < 3; ++c) raw[c] += p->preflash_raw[c] * p->preflash;
        lc[i] = (fmaxf(raw[0], 0.0f) + 1e-10f) * outer;
        lm[i] = (fmaxf(raw[1], 0.0f) + 1e-10f) * outer;
        ly[i] = (fmaxf(raw[2], 0.0f) + 1e-10f) * outer;
    }
    free(pk.lut_store);
    return 0;
}

/* Print density C, M, Y from the diffused print-linear exposure: log10(max(v, 0) +
 * 1e-10) on the print curves (:1449-1488, src/Cuda/JuicerCudaDeviceHelpers.cuh:1025). */
int oracle_enlarger_develop(const FjPreparedHostData* h, const float* lc, const float* lm, const float* ly, int W,
                            int H, float* dc, float* dm, float* dy) {
    Packed pk;
    if (pack(h, &pk) || !pk.p.print) {
        free(pk.lut_store);
        return 1;
    }
    const Pack* p = &pk.p;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)W * H; ++i) {
        const float v[3] = {lc[i], lm[i], ly[i]};
        float* out[3] = {dc, dm, dy};
        for (int c = 0; c < 3; ++c) out[c][i] = curve_at(&p->pdc[c], log10f(fmaxf(v[c], 0.0f) + 1e-10f), 1.0f);
    }
    free(pk.lut_store);
    return 0;
}

/* ------------------------------------------------------------------------------ *
 * Visual grain (a15). Restates src/Cuda/Film/JuicerCudaFilmPipeline.cu:1580-2986  *
 * (random draws, particle model, Wang offsets, value noise, breathing, clump,     *
 * frame uniforms, layer lookup, sample kernels) and the schedule of               *
 * src/Cuda/Scan/JuicerCudaScanPipeline.cu:3141-3740 with its blurs (:317-380,     *
 * :454-578). The reference's compiler contracts a + b * c into one fused          *
 * multiply-add; those places use fmaf() here. expf/logf/cosf/sinf/sqrtf/rsqrtf    *
 * come from libm (rsqrtf as 1/sqrtf), so the oracle agrees with a GPU to the      *
 * last bits of those functions: the random streams themselves (blue-noise         *
 * lookups, Philox words, hashes) are exact.                                        *
 * ------------------------------------------------------------------------------ */

typedef struct {
    int breathing_active;
    float breathing_t;
    uint64_t seed_a, seed_b;
    float cell_small, cell_large, drift_x, drift_y, roll_y, mix;
    int clump_active;
    float clump_cell, clump_roll;
    uint64_t clump_seed;
    float clump_rms, clump_mu, clump_sigma;
} OGrainUniforms;

typedef struct {
    const FjVisualGrain* g;
    const uint8_t* stbn;
    int stbn_w, stbn_h, stbn_frames, stbn_off_x, stbn_off_y, stbn_frame;
    const uint8_t* wang;
    const uint8_t* wang_lut;
    int wang_w, wang_h, wang_count, wang_colors;
    const float* base[3];
    const float* layer[3][3];
    int n;
    int positive;
    /* per-scale overrides */
    uint64_t seed, seed_next;
    float n_particles[3], od_particle[3], n_layers[3][3], od_layers[3][3];
    OGrainUniforms u;
} OGrain;

static inline uint64_t og_splitmix(uint64_t v) {
    v += 0x9E3779B97F4A7C15ULL;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}
static inline int og_wrap(int64_t c, int size) {
    if (size <= 0) return 0;
    if ((size & (size - 1)) == 0) return (int)((uint64_t)c & (uint64_t)(size - 1));
    c %= (int64_t)size;
    if (c < 0) c += size;
    return (int)c;
}
static inline float og_clamp(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
static inline float og_san(float v) { return isfinite(v) ? v : 0.0f; }
static inline float og_smooth(float t) { return (t * t) * fmaf(-2.0f, t, 3.0f); }
static inline float og_hash01(int x, int y, uint64_t seed) {
    uint64_t h = og_splitmix(seed ^ ((uint64_t)(int64_t)x * 0x9E3779B97F4A7C15ULL) ^
                             ((uint64_t)(int64_t)y * 0xBF58476D1CE4E5B9ULL));
    return (float)(uint32_t)(h & 0xFFFFFFFFu) * (1.0f / 4294967296.0f);
}
static inline float og_spatial(int x, int y, uint64_t seed) {
    uint32_t lo = (uint32_t)seed, hi = (uint32_t)(seed >> 32);
    uint32_t h = lo ^ ((hi << 16) | (hi >> 16));
    h ^= (uint32_t)x * 0x9E3779B9u;
    h ^= (uint32_t)y * 0x85EBCA6Bu;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return (float)h * (1.0f / 4294967296.0f);
}
static inline float og_noise(float cx, float cy, uint64_t seed) {
    int ix = (int)floorf(cx), iy = (int)floorf(cy);
    float sx = og_smooth(cx - (float)ix), sy = og_smooth(cy - (float)iy);
    float v00 = og_spatial(ix, iy, seed), v10 = og_spatial(ix + 1, iy, seed);
    float v01 = og_spatial(ix, iy + 1, seed), v11 = og_spatial(ix + 1, iy + 1, seed);
    float v0 = fmaf(v10 - v00, sx, v00), v1 = fmaf(v11 - v01, sx, v01);
    return fmaf(v1 - v0, sy, v0);
}

/* Philox4x32-10, openrand arrangement (third_party/openrand/philox.h:60-150). */
typedef struct {
    uint32_t k0, k1, c0, c1, c2, n;
} OPhilox;
static uint32_t og_philox(OPhilox* p) {
    uint32_t x0 = p->c0, x1 = p->c1, x2 = p->c2, x3 = p->n, a = p->k0, b = p->k1;
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            a += 0x9E3779B9u;
            b += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * x0, p1 = (uint64_t)0xCD9E8D57u * x2;
        uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ a, y2 = (uint32_t)(p0 >> 32) ^ x3 ^ b;
        x0 = y0;
        x1 = (uint32_t)p1;
        x2 = y2;
        x3 = (uint32_t)p0;
    }
    p->n++;
    return x0;
}

typedef struct {
    OPhilox ph;
    const OGrain* o;
    uint64_t ax, ay, seed;
    uint32_t draw;
    int stbn, wx, wy, mask_w, mask_h;
    int64_t pitch;
    size_t row_base;
} ORng;

static void og_rng_init(ORng* r, const OGrain* o, uint64_t seed, uint64_t ax, uint64_t ay, int stbn, int frame_off,
                        int wx, int wy) {
    memset(r, 0, sizeof(*r));
    r->ph.k0 = (uint32_t)(seed >> 32);
    r->ph.k1 = (uint32_t)seed;
    r->ph.c0 = (uint32_t)ax;
    r->ph.c1 = (uint32_t)ay;
    r->ph.c2 = 0xAAAAAAAAu;
    r->o = o;
    r->ax = ax;
    r->ay = ay;
    r->seed = seed;
    r->stbn = stbn;
    r->wx = wx;
    r->wy = wy;
    r->mask_w = r->mask_h = -1;
    if (!stbn) return;
    if ((o->stbn_w & (o->stbn_w - 1)) == 0 && (o->stbn_h & (o->stbn_h - 1)) == 0) {
        r->mask_w = o->stbn_w - 1;
        r->mask_h = o->stbn_h - 1;
    }
    if (o->g->pitch_px > 0) r->pitch = (int64_t)o->g->pitch_px * (o->g->frame0 + (int64_t)frame_off);
    r->row_base = (size_t)og_wrap((int64_t)o->stbn_frame + frame_off, o->stbn_frames) * (size_t)o->stbn_h;
}

static float og_uniform(ORng* r) {
    if (r->stbn) {
        uint32_t d = r->draw++;
        uint64_t h = og_splitmix(r->seed + (uint64_t)d * 0x9E3779B97F4A7C15ULL);
        int ox = (int)(h & 0xFFFFu) + r->wx, oy = (int)((h >> 16) & 0xFFFFu) + r->wy;
        int64_t xc = (int64_t)r->ax + ox + r->o->stbn_off_x;
        int64_t yc = (int64_t)r->ay + oy + r->o->stbn_off_y + r->pitch;
        int x, y;
        if (r->mask_w >= 0) {
            x = (int)((uint64_t)xc & (uint64_t)r->mask_w);
            y = (int)((uint64_t)yc & (uint64_t)r->mask_h);
        } else {
            x = og_wrap(xc, r->o->stbn_w);
            y = og_wrap(yc, r->o->stbn_h);
        }
        uint8_t v = r->o->stbn[(r->row_base + (size_t)y) * (size_t)r->o->stbn_w + (size_t)x];
        return ((float)v + 0.5f) * (1.0f / 256.0f);
    }
    return fmaf((float)og_philox(&r->ph), 1.0f / 4294967296.0f, 0.5f / 4294967296.0f);
}

static float og_normal(ORng* r) {
    float u1 = og_clamp(og_uniform(r), 1e-7f, 1.0f);
    float u2 = og_uniform(r);
    return sqrtf(-2.0f * logf(u1)) * cosf(6.28318530717958647692f * u2);
}

static int og_poisson(float lambda, ORng* r) {
    if (!isfinite(lambda) || !(lambda > 0.0f)) return 0;
    if (lambda < 10.0f) {
        float L = expf(-lambda), p = 1.0f;
        int k = 0;
        while (p > L && k < 1024) {
            ++k;
            p *= og_clamp(og_uniform(r), 1e-7f, 1.0f);
        }
        return k - 1;
    }
    float z = og_normal(r);
    float s = fmaf(sqrtf(lambda), z, lambda);
    if (!isfinite(s)) s = 0.0f;
    int k = (int)floorf(s + 0.5f);
    return k < 0 ? 0 : k;
}

static float og_particle(const OGrain* o, float density, float dmax, float np, float od, float unif, uint64_t seed,
                         int frame_off, uint64_t ax, uint64_t ay, int stbn, int wx, int wy) {
    if (!isfinite(density) || density < 0.0f) density = 0.0f;
    float p = og_clamp(density / dmax, 1e-6f, 1.0f - 1e-6f);
    float u = isfinite(unif) ? og_clamp(unif, 0.0f, 1.0f) : 0.0f;
    float sat = fmaf(-(p * u), 1.0f - 1e-6f, 1.0f);
    if (!isfinite(sat) || sat <= 0.0f) sat = 1e-6f;
    ORng r;
    og_rng_init(&r, o, seed, ax, ay, stbn, frame_off, wx, wy);
    float lambda = np / sat;
    int count = og_poisson(lambda * p, &r);
    return og_san((float)count * od * sat);
}

static void og_wang(const OGrain* o, uint64_t ax, uint64_t ay, int* ox, int* oy) {
    const FjVisualGrain* g = o->g;
    *ox = *oy = 0;
    if (!o->wang || !o->wang_lut || o->wang_w <= 0 || o->wang_h <= 0 || o->wang_count <= 0) return;
    if (!(g->pixel_size_um > 0.0f) || !(g->wang_cell_mm > 0.0f) || o->wang_colors <= 0) return;
    float xmm = (float)ax * (g->pixel_size_um * 0.001f), ymm = (float)ay * (g->pixel_size_um * 0.001f);
    float inv = 1.0f / g->wang_cell_mm;
    float cx = xmm * inv, cy = ymm * inv;
    float fx = cx - floorf(cx), fy = cy - floorf(cy);
    int64_t mx = (int64_t)floorf(cx), my = (int64_t)floorf(cy);
    uint64_t s0 = g->clip_token != 0 ? g->clip_token : g->session_seed;
    uint64_t base = s0 != 0 ? s0 : 1ULL;
#define OG_HU32(X, Y, SALT)                                                                                        \
    ((uint32_t)(og_splitmix(base ^ (SALT) ^ ((uint64_t)(int64_t)(X) * 0x9E3779B97F4A7C15ULL) ^                    \
                            ((uint64_t)(int64_t)(Y) * 0xBF58476D1CE4E5B9ULL)) &                                    \
                0xFFFFFFFFu))
    uint32_t colors = (uint32_t)o->wang_colors;
    uint32_t l = OG_HU32((int)mx, (int)my, 0xA5A5A5A5ULL) % colors;
    uint32_t rr = OG_HU32((int)(mx + 1), (int)my, 0x5A5A5A5AULL) % colors;
    uint32_t t = OG_HU32((int)mx, (int)my, 0xC3C3C3C3ULL) % colors;
    uint32_t b = OG_HU32((int)mx, (int)(my + 1), 0x3C3C3C3CULL) % colors;
#undef OG_HU32
    size_t c = colors;
    int tile = (int)o->wang_lut[(((size_t)l * c + rr) * c + t) * c + b];
    int w = o->wang_w, h = o->wang_h;
    int tx = (int)floorf(fx * (float)w), ty = (int)floorf(fy * (float)h);
    if (tx >= w) tx = w - 1;
    if (ty >= h) ty = h - 1;
    float v[2];
    int xs[2] = {tx, (tx + (w >> 1)) % w}, ys[2] = {ty, (ty + (h >> 1)) % h};
    for (int i = 0; i < 2; ++i) {
        if (tile < 0 || tile >= o->wang_count) {
            v[i] = 0.0f;
            continue;
        }
        int x = xs[i] < 0 ? 0 : (xs[i] >= w ? w - 1 : xs[i]);
        int y = ys[i] < 0 ? 0 : (ys[i] >= h ? h - 1 : ys[i]);
        v[i] = ((float)o->wang[((size_t)tile * h + y) * w + x] + 0.5f) * (1.0f / 256.0f);
    }
    int warp_x = o->stbn_w > 0 ? ((o->stbn_w / 8) > 4 ? o->stbn_w / 8 : 4) : 0;
    int warp_y = o->stbn_h > 0 ? ((o->stbn_h / 8) > 4 ? o->stbn_h / 8 : 4) : 0;
    if (warp_x == 0 || warp_y == 0) return;
    *ox = (int)floorf((v[0] - 0.5f) * 2.0f * (float)warp_x);
    *oy = (int)floorf((v[1] - 0.5f) * 2.0f * (float)warp_y);
}

static float og_breathing(const OGrain* o, uint64_t ax, uint64_t ay) {
    const OGrainUniforms* u = &o->u;
    if (!u->breathing_active) return 1.0f;
    float bx = (float)ax + u->drift_x, by = (float)ay + u->drift_y + u->roll_y;
    float xs = bx / u->cell_small, ys = by / u->cell_small, xl = bx / u->cell_large, yl = by / u->cell_large;
    float sa = og_noise(xs, ys, u->seed_a ^ 0x9E3779B97F4A7C15ULL), sb = og_noise(xs, ys, u->seed_b ^ 0x9E3779B97F4A7C15ULL);
    float la = og_noise(xl, yl, u->seed_a ^ 0xBF58476D1CE4E5B9ULL), lb = og_noise(xl, yl, u->seed_b ^ 0xBF58476D1CE4E5B9ULL);
    float ns = fmaf(sb - sa, u->breathing_t, sa), nl = fmaf(lb - la, u->breathing_t, la);
    float noise = fmaf(u->mix, ns, (1.0f - u->mix) * nl);
    float f = fmaf(o->g->breathing_amplitude, fmaf(noise, 2.0f, -1.0f), 1.0f);
    return f > 0.0f ? f : 0.0f;
}

static float og_clump(const OGrain* o, uint64_t ax, uint64_t ay) {
    const OGrainUniforms* u = &o->u;
    if (!u->clump_active) return 1.0f;
    float xs = (float)ax / u->clump_cell, ys = ((float)ay + u->clump_roll) / u->clump_cell;
    float a = og_noise(xs, ys, u->clump_seed ^ 0x9E3779B97F4A7C15ULL);
    float b = og_noise(xs + 19.19f, ys + 7.23f, u->clump_seed ^ 0xBF58476D1CE4E5B9ULL);
    float u1 = og_clamp(a, 1e-6f, 1.0f - 1e-6f), u2 = og_clamp(b, 0.0f, 1.0f);
    float n = sqrtf(-2.0f * logf(u1)) * cosf(6.28318530717958647692f * u2);
    float v = expf(fmaf(u->clump_sigma, n, u->clump_mu));
    if (!isfinite(v)) v = 1.0f;
    return v * u->clump_rms;
}

static void og_lognormal(float mean, float sd, float* mu, float* sigma) {
    float m2 = mean * mean, s2 = sd * sd;
    float sq = logf(1.0f + s2 / m2);
    *sigma = sqrtf(fmaxf(0.0f, sq));
    *mu = fmaf(-0.5f, sq, logf(fmaxf(1e-12f, mean)));
}

static void og_uniforms(OGrain* o) {
    const FjVisualGrain* g = o->g;
    OGrainUniforms u;
    memset(&u, 0, sizeof(u));
    float time = (float)g->frame0 + g->frame_alpha;
    if (g->breathing_amplitude > 0.0f && g->breathing_period_frames > 0 && g->pixel_size_um > 0.0f &&
        g->breathing_cell_um_small > 0.0f && g->breathing_cell_um_large > 0.0f) {
        float period = (float)g->breathing_period_frames;
        float step_f = floorf(time / period);
        int64_t step = (int64_t)step_f;
        float frac = fmaf(-step_f, period, time) / period;
        u.breathing_t = og_smooth(og_clamp(frac, 0.0f, 1.0f));
        uint64_t seed = g->session_seed != 0 ? g->session_seed : 1ULL;
        u.seed_a = og_splitmix(seed ^ ((uint64_t)step * 0x8EBC6AF09C88C6E3ULL));
        u.seed_b = og_splitmix(seed ^ ((uint64_t)(step + 1) * 0x8EBC6AF09C88C6E3ULL));
        float inv = 1.0f / g->pixel_size_um;
        u.cell_small = fmaxf(4.0f, g->breathing_cell_um_small * inv);
        u.cell_large = fmaxf(4.0f, g->breathing_cell_um_large * inv);
        float drift = g->breathing_drift_um_per_frame > 0.0f ? g->breathing_drift_um_per_frame * inv : 0.0f;
        float dx = 0.0f, dy = 0.0f;
        if (drift > 0.0f) {
            uint64_t h = og_splitmix(seed ^ 0x6A09E667F3BCC909ULL);
            float angle = (float)(uint32_t)(h & 0xFFFFFFFFu) * (1.0f / 4294967296.0f) * 6.28318530717958647692f;
            dx = cosf(angle) * drift;
            dy = sinf(angle) * drift;
        }
        float roll = g->pitch_px > 0 ? (float)g->pitch_px : 0.0f;
        u.drift_x = dx * time;
        u.drift_y = dy * time;
        u.roll_y = roll * time;
        u.mix = og_clamp(g->breathing_mix, 0.0f, 1.0f);
        u.breathing_active = 1;
    }
    float sds = g->micro_structure[1] * 0.001f;
    if (sds > 0.0f && g->pixel_size_um > 0.0f) {
        float cell = g->micro_structure[0];
        if (!(cell > 0.0f)) cell = 0.0f;
        float inv = 1.0f / g->pixel_size_um;
        u.clump_cell = cell * inv;
        if (!(u.clump_cell > 4.0f)) u.clump_cell = 4.0f;
        float roll = g->pitch_px > 0 ? (float)g->pitch_px : 0.0f;
        u.clump_roll = roll * time;
        u.clump_seed = g->clip_token != 0 ? g->clip_token : g->session_seed;
        if (u.clump_seed == 0) u.clump_seed = 1ULL;
        float sd = sds;
        u.clump_rms = 1.0f;
        float mix = og_clamp(g->clump_temporal_mix, 0.0f, 1.0f);
        if (mix > 0.0f) {
            int per = g->clump_morph_period_frames;
            if (per <= 0) per = 1;
            float period = (float)per;
            float step_f = floorf(time / period);
            int64_t step = (int64_t)step_f;
            float frac = fmaf(-step_f, period, time) / period;
            float t = og_smooth(og_clamp(frac, 0.0f, 1.0f));
            uint64_t ts = g->session_seed != 0 ? g->session_seed : 1ULL;
            uint64_t sa = og_splitmix(ts ^ ((uint64_t)step * 0xD2B74407B1CE6E93ULL));
            uint64_t sb = og_splitmix(ts ^ ((uint64_t)(step + 1) * 0xD2B74407B1CE6E93ULL));
            float u1a = og_hash01(0, 0, sa ^ 0x9E3779B97F4A7C15ULL), u2a = og_hash01(1, 0, sa ^ 0xBF58476D1CE4E5B9ULL);
            float u1b = og_hash01(0, 0, sb ^ 0x9E3779B97F4A7C15ULL), u2b = og_hash01(1, 0, sb ^ 0xBF58476D1CE4E5B9ULL);
            float u1 = og_clamp(fmaf(u1b - u1a, t, u1a), 1e-6f, 1.0f - 1e-6f);
            float u2 = og_clamp(fmaf(u2b - u2a, t, u2a), 0.0f, 1.0f);
            float nt = sqrtf(-2.0f * logf(u1)) * cosf(6.28318530717958647692f * u2);
            float ssd = mix * 0.23597824f, mu, sigma;
            og_lognormal(1.0f, ssd, &mu, &sigma);
            float strength = expf(fmaf(sigma, nt, mu));
            strength *= 1.0f / sqrtf(fmaf(ssd, ssd, 1.0f));
            sd = sds * strength;
            float den = fmaf(sd, sd, 1.0f), num = fmaf(sds, sds, 1.0f);
            u.clump_rms = den > 0.0f ? sqrtf(num / den) : 1.0f;
        }
        og_lognormal(1.0f, sd, &u.clump_mu, &u.clump_sigma);
        u.clump_active = 1;
    }
    o->u = u;
}

static float og_layer_density(const OGrain* o, int ch, int layer, float density) {
    const float* x = o->base[ch];
    const float* y = o->layer[layer][ch];
    int n = o->n;
    if (!x || !y || n <= 0) return density;
    if (!isfinite(density)) return y[0];
    int pos = o->positive;
    float q = pos ? -density : density;
#define OG_AX(i) (pos ? -x[(i)] : x[(i)])
    int bounded = (o->g->flags & (FJ_GRAIN_AXIS_FINITE_C << ch)) != 0 && n == 256;
    int b0 = 0, b1 = n - 1;
    if (!bounded) {
        while (b0 < n && !isfinite(OG_AX(b0))) ++b0;
        if (b0 >= n) return density;
        while (b1 > b0 && !isfinite(OG_AX(b1))) --b1;
    }
    float xmin = OG_AX(b0), xmax = OG_AX(b1);
    if (!isfinite(xmin) || !isfinite(xmax) || !(xmax >= xmin)) return y[b0];
    if (q <= xmin) return y[b0];
    if (q >= xmax) return y[b1];
    int i1 = b0 + 1;
    if (bounded) {
        const float* prefix = o->g->layer_axis_block_prefix_max[ch];
        int lo = 0, hi = 15;
        for (int s = 0; s < 4; ++s) {
            int mid = lo + (hi - lo) / 2;
            if (prefix[mid] < q)
                lo = mid + 1;
            else
                hi = mid;
        }
        i1 = lo * 16 > 1 ? lo * 16 : 1;
        int end = (lo + 1) * 16 - 1 < b1 ? (lo + 1) * 16 - 1 : b1;
        while (i1 <= end && OG_AX(i1) < q) ++i1;
    } else {
        while (i1 <= b1 && OG_AX(i1) < q) ++i1;
    }
    if (i1 > b1) return y[b1];
    int i0 = i1 - 1;
    float x0 = OG_AX(i0), x1 = OG_AX(i1), den = x1 - x0;
#undef OG_AX
    if (!(den > 0.0f) || !isfinite(den)) return y[i0];
    return fmaf((q - x0) / den, y[i1] - y[i0], y[i0]);
}

static float og_modulate(float g, float density, float br, float cl) { return fmaf((g - density) * br, cl, density); }

static float og_retime(float g, float gn, float density, float alpha) {
    float d0 = g - density, d1 = gn - density;
    float blend = fmaf(d1 - d0, alpha, d0);
    float w0 = 1.0f - alpha;
    float den = fmaf(w0, w0, alpha * alpha) + 1e-6f;
    return fmaf(blend, 1.0f / sqrtf(den), density);
}

/* mode 0 simple, 1 layer, 2 triplet: the sanitised sample of one pixel. */
static float og_sample(const OGrain* o, int mode, int ch, int layer, float in_density, uint64_t ax, uint64_t ay) {
    const FjVisualGrain* g = o->g;
    int stbn = (o->stbn && o->stbn_w > 0 && o->stbn_h > 0 && o->stbn_frames > 0) ? 1 : 0;
    float alpha = g->frame_alpha;
    int retime = alpha > 1e-6f && alpha < 0.999999f;
    int wx = 0, wy = 0;
    float cl = og_clump(o, ax, ay);
    if (stbn) og_wang(o, ax, ay, &wx, &wy);
    float br = og_breathing(o, ax, ay);
    if (mode == 0) {
        float density = in_density + g->particle_density_min_cmy[ch];
        int nsub = g->sublayer_count > 0 ? (int)g->sublayer_count : 1;
        float acc = 0.0f, accn = 0.0f;
        for (int sl = 0; sl < nsub; ++sl) {
            uint64_t salt = (uint64_t)ch + (uint64_t)sl * 10ULL;
            acc += og_particle(o, density, g->density_max_cmy[ch], o->n_particles[ch], o->od_particle[ch],
                               g->uniformity_cmy[ch], o->seed ^ salt, 0, ax, ay, stbn, wx, wy);
            if (retime)
                accn += og_particle(o, density, g->density_max_cmy[ch], o->n_particles[ch], o->od_particle[ch],
                                    g->uniformity_cmy[ch], o->seed_next ^ salt, 1, ax, ay, stbn, wx, wy);
        }
        acc /= (float)nsub;
        if (retime) accn /= (float)nsub;
        acc = og_modulate(acc, density, br, cl);
        if (retime) acc = og_retime(acc, og_modulate(accn, density, br, cl), density, alpha);
        return og_san(acc);
    }
    float sum = 0.0f;
    for (int l = (mode == 1 ? layer : 0); l < (mode == 1 ? layer + 1 : 3); ++l) {
        float density = og_layer_density(o, ch, l, in_density) + g->density_min_layers[l][ch];
        uint64_t salt = (uint64_t)ch + (uint64_t)l * 10ULL;
        float v = og_particle(o, density, g->density_max_layers[l][ch], o->n_layers[l][ch], o->od_layers[l][ch],
                              g->uniformity_cmy[ch], o->seed ^ salt, 0, ax, ay, stbn, wx, wy);
        v = og_modulate(v, density, br, cl);
        if (retime) {
            float vn = og_particle(o, density, g->density_max_layers[l][ch], o->n_layers[l][ch], o->od_layers[l][ch],
                                   g->uniformity_cmy[ch], o->seed_next ^ salt, 1, ax, ay, stbn, wx, wy);
            v = og_retime(v, og_modulate(vn, density, br, cl), density, alpha);
        }
        if (mode == 1) return og_san(v);
        sum += og_san(v);
    }
    return og_san(sum);
}

static int og_reflect_half(long i, int n) {
    if (n <= 1) return 0;
    long p = 2L * n, m = i % p;
    if (m < 0) m += p;
    return (int)(m < n ? m : p - 1 - m);
}

/* Normalised Gaussian taps (rust/film-juicer-core/src/optics/gaussian.rs:16-52). */
static void og_taps(int radius, float sigma, float* w) {
    double s = (double)sigma, s2 = s * s * 2.0, sum = 0.0;
    for (int i = -radius; i <= radius; ++i) {
        double v = exp(-((double)i * (double)i) / s2);
        w[i + radius] = (float)v;
        sum += v;
    }
    double rec = sum != 0.0 ? 1.0 / sum : 0.0;
    for (int i = 0; i <= 2 * radius; ++i) w[i] = (float)((double)w[i] * rec);
}

static void og_blur_rows(const float* in, float* out, const float* w, int r, int W, int H) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float acc = 0.0f;
            for (int k = 0; k <= 2 * r; ++k) acc = fmaf(in[(size_t)y * W + og_reflect_half((long)x - r + k, W)], w[k], acc);
            out[(size_t)y * W + x] = og_san(acc);
        }
}

static float og_blur_col(const float* in, const float* w, int r, int W, int H, int x, int y) {
    float acc = 0.0f;
    for (int k = 0; k <= 2 * r; ++k) acc = fmaf(in[(size_t)og_reflect_half((long)y - r + k, H) * W + x], w[k], acc);
    return og_san(acc);
}

typedef struct {
    float w[151];
    int r;
    uint64_t hash;
} OTaps;

typedef struct {
    OGrain o;
    OTaps corr[3], dye[3][3];
    int W, H;
    float *temp, *scale, *layer;
} OSched;

/* One scale of one channel, accumulated into `target` (generate_scale). */
static int og_scale_pass(OSched* s, const float* dens, int ch, uint64_t salt, float factor, const OTaps* corr,
                         int apply, float weight, int init, float* target) {
    OGrain* o = &s->o;
    const FjVisualGrain* g = o->g;
    int W = s->W, H = s->H;
    size_t N = (size_t)W * H;
    o->seed = g->seed_base ^ salt;
    o->seed_next = g->seed_base_next ^ salt;
    for (int c = 0; c < 3; ++c) {
        o->n_particles[c] = g->n_particles_cmy[c] / factor;
        o->od_particle[c] = g->od_particle_cmy[c] * factor;
        for (int l = 0; l < 3; ++l) {
            o->n_layers[l][c] = g->n_particles_layers[l][c] / factor;
            o->od_layers[l][c] = g->od_particle_layers[l][c] * factor;
        }
    }
    float bias = -g->particle_density_min_cmy[ch];
    int sub = (g->flags & FJ_GRAIN_SUBLAYERS) != 0;
    int delta_formed = 0;
#define OG_DELTA(v, i)                                                                                             \
    do {                                                                                                            \
        if (bias != 0.0f) (v) = og_san((v) + bias);                                                               \
        (v) = og_san((v) - dens[(i)]);                                                                              \
    } while (0)
    if (sub) {
        const OTaps *d0 = &s->dye[0][ch], *d1 = &s->dye[1][ch], *d2 = &s->dye[2][ch];
        int zero = d0->r <= 0 && d1->r <= 0 && d2->r <= 0;
        int same = d0->r == d1->r && d0->r == d2->r && (zero || (d0->hash == d1->hash && d0->hash == d2->hash));
        if (same) {
#pragma omp parallel for schedule(dynamic, 4)
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    size_t i = (size_t)y * W + x;
                    float v = og_sample(o, 2, ch, 0, dens[i], (uint64_t)((int64_t)g->render_extent.x + x),
                                        (uint64_t)((int64_t)g->render_extent.y + y));
                    if (zero) {
                        v = og_san(0.0f + v);
                        OG_DELTA(v, i);
                        s->scale[i] = v;
                    } else {
                        s->layer[i] = v;
                    }
                }
            if (!zero) {
                og_blur_rows(s->layer, s->temp, d0->w, d0->r, W, H);
#pragma omp parallel for schedule(static)
                for (int y = 0; y < H; ++y)
                    for (int x = 0; x < W; ++x) {
                        size_t i = (size_t)y * W + x;
                        float v = og_san(0.0f + og_blur_col(s->temp, d0->w, d0->r, W, H, x, y));
                        OG_DELTA(v, i);
                        s->scale[i] = v;
                    }
            }
            delta_formed = 1;
        } else {
            for (int l = 0; l < 3; ++l) {
                const OTaps* d = &s->dye[l][ch];
#pragma omp parallel for schedule(dynamic, 4)
                for (int y = 0; y < H; ++y)
                    for (int x = 0; x < W; ++x) {
                        size_t i = (size_t)y * W + x;
                        float v = og_sample(o, 1, ch, l, dens[i], (uint64_t)((int64_t)g->render_extent.x + x),
                                            (uint64_t)((int64_t)g->render_extent.y + y));
                        if (d->r > 0) {
                            s->layer[i] = v;
                        } else {
                            v = og_san((l == 0 ? 0.0f : s->scale[i]) + v);
                            if (l == 2) OG_DELTA(v, i);
                            s->scale[i] = v;
                        }
                    }
                if (d->r > 0) {
                    og_blur_rows(s->layer, s->temp, d->w, d->r, W, H);
#pragma omp parallel for schedule(static)
                    for (int y = 0; y < H; ++y)
                        for (int x = 0; x < W; ++x) {
                            size_t i = (size_t)y * W + x;
                            float v = og_san((l == 0 ? 0.0f : s->scale[i]) + og_blur_col(s->temp, d->w, d->r, W, H, x, y));
                            if (l == 2) OG_DELTA(v, i);
                            s->scale[i] = v;
                        }
                }
            }
            delta_formed = 1;
        }
    } else {
#pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                size_t i = (size_t)y * W + x;
                float v = og_sample(o, 0, ch, 0, dens[i], (uint64_t)((int64_t)g->render_extent.x + x),
                                    (uint64_t)((int64_t)g->render_extent.y + y));
                OG_DELTA(v, i);
                s->scale[i] = v;
            }
        delta_formed = 1;
    }
#undef OG_DELTA
    if (!delta_formed) return 1;
    float wgt = isfinite(weight) ? weight : 0.0f;
    if (apply && corr->r > 0) {
        og_blur_rows(s->scale, s->temp, corr->w, corr->r, W, H);
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                size_t i = (size_t)y * W + x;
                target[i] = og_san(fmaf(wgt, og_blur_col(s->temp, corr->w, corr->r, W, H, x, y), init ? 0.0f : target[i]));
            }
    } else {
        for (size_t i = 0; i < N; ++i) target[i] = og_san(fmaf(wgt, s->scale[i], init ? 0.0f : target[i]));
    }
    return 0;
}

static int og_mix(OSched* s, const float* dens, int ch, float* target) {
    const FjVisualGrain* g = s->o.g;
    float wf = g->size_mix_weights[0], wm = g->size_mix_weights[1], wc = g->size_mix_weights[2];
    float sms = g->size_mix_scale;
    float ws[3] = {wf, wm, wc}, fac[3] = {1.0f, sqrtf(sms), sms};
    uint64_t salts[3] = {0xA24BAED4963EE407ULL, 0x9F6C1E6B2C4D7A13ULL, 0x3C79AC492BA7B653ULL};
    int init = 1;
    for (int i = 0; i < 3; ++i) {
        if (!(ws[i] > 0.0f)) continue;
        int apply = i == 0 ? s->corr[0].r > 0 : 1;
        if (og_scale_pass(s, dens, ch, salts[i], fac[i], &s->corr[i], apply, ws[i], init, target)) return 1;
        init = 0;
    }
    float gain = isfinite(g->size_mix_gain) ? g->size_mix_gain : 0.0f;
    size_t N = (size_t)s->W * s->H;
    for (size_t i = 0; i < N; ++i) target[i] = og_san(target[i] * gain);
    return 0;
}

static uint64_t og_fnv(uint64_t a, uint64_t b) {
    uint64_t h = 0xcbf29ce484222325ULL, v[2] = {a, b};
    for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 8; ++i) {
            h ^= (v[k] >> (8 * i)) & 0xFFu;
            h *= 0x100000001b3ULL;
        }
    return h;
}

/* Visual grain on the three density planes in place. `noise` may be NULL (Philox
 * stream); base curves are the capture density curves of C, M, Y (n samples), layer
 * curves [layer][CMY]. Returns 0 on success. */
int oracle_visual_grain(const FjVisualGrain* g, const FjStaticNoise* noise, const float* const* base_cmy,
                        const float* const* layers, int n, int positive, float* dc, float* dm, float* dy, int W, int H) {
    if (!(g->flags & FJ_GRAIN_ACTIVE)) return 0;
    OSched s;
    memset(&s, 0, sizeof(s));
    OGrain* o = &s.o;
    o->g = g;
    if (noise) {
        o->stbn = noise->stbn.data;
        o->stbn_w = noise->stbn_width;
        o->stbn_h = noise->stbn_height;
        o->stbn_frames = noise->stbn_frames;
        o->wang = noise->wang_tiles.data;
        o->wang_lut = noise->wang_lut.data;
        o->wang_w = noise->wang_width;
        o->wang_h = noise->wang_height;
        o->wang_count = (int)noise->wang_tile_count;
        o->wang_colors = noise->wang_colors;
    }
    o->stbn_off_x = o->stbn_w > 0 ? (int)(og_fnv(g->session_seed, 0xA5u) % (uint64_t)o->stbn_w) : 0;
    o->stbn_off_y = o->stbn_h > 0 ? (int)(og_fnv(g->session_seed, 0x5Au) % (uint64_t)o->stbn_h) : 0;
    if (o->stbn_frames > 0) {
        int64_t ph = (int64_t)(g->session_seed % (uint64_t)o->stbn_frames);
        int f = (int)((g->frame0 + ph) % o->stbn_frames);
        o->stbn_frame = f < 0 ? f + o->stbn_frames : f;
    }
    int sub = (g->flags & FJ_GRAIN_SUBLAYERS) != 0;
    if (sub) {
        for (int c = 0; c < 3; ++c) {
            o->base[c] = base_cmy[c];
            for (int l = 0; l < 3; ++l) o->layer[l][c] = layers[l * 3 + c];
        }
        o->n = n;
    }
    o->positive = positive;
    for (int i = 0; i < 3; ++i)
        if (g->correlation[i].radius > 0) {
            s.corr[i].r = g->correlation[i].radius;
            s.corr[i].hash = g->correlation[i].hash;
            og_taps(s.corr[i].r, g->correlation[i].sigma_px, s.corr[i].w);
        }
    for (int l = 0; l < 3; ++l)
        for (int c = 0; c < 3; ++c)
            if (sub && g->dye_cloud[l][c].radius > 0) {
                s.dye[l][c].r = g->dye_cloud[l][c].radius;
                s.dye[l][c].hash = g->dye_cloud[l][c].hash;
                og_taps(s.dye[l][c].r, g->dye_cloud[l][c].sigma_px, s.dye[l][c].w);
            }
    s.W = W;
    s.H = H;
    size_t N = (size_t)W * H;
    float* buf = (float*)calloc(5 * N, sizeof(float));
    if (!buf) return 1;
    s.temp = buf;
    s.scale = buf + N;
    s.layer = buf + 2 * N;
    float* accum = buf + 3 * N;
    float* shared = buf + 4 * N;
    float* dens[3] = {dc, dm, dy};
    int rc = 0;
    unsigned debug = g->debug_view;
    if (debug == FJ_GRAIN_DEBUG_MEAN_DENSITY) {
        float sc = g->debug_scale * 4.0f;
        sc = isfinite(sc) ? sc : 1.0f;
        for (size_t i = 0; i < N; ++i) {
            float a = (dc[i] + dm[i] + dy[i]) * (1.0f / 3.0f);
            if (!isfinite(a)) a = 0.0f;
            dc[i] = dm[i] = dy[i] = fmaf(a, sc, 0.0f);
        }
        free(buf);
        return 0;
    }
    og_uniforms(o);
    if (debug >= FJ_GRAIN_DEBUG_DELTA_FINE && debug <= FJ_GRAIN_DEBUG_DELTA_COARSE_RAW) {
        int coarse = debug == FJ_GRAIN_DEBUG_DELTA_COARSE || debug == FJ_GRAIN_DEBUG_DELTA_COARSE_RAW;
        int raw = debug == FJ_GRAIN_DEBUG_DELTA_FINE_RAW || debug == FJ_GRAIN_DEBUG_DELTA_COARSE_RAW;
        for (int c = 0; c < 3 && !rc; ++c) {
            if (!coarse || g->size_mix_weights[2] > 0.0f) {
                const OTaps* corr = coarse ? &s.corr[2] : &s.corr[0];
                rc = og_scale_pass(&s, dens[c], c, coarse ? 0x3C79AC492BA7B653ULL : 0xA24BAED4963EE407ULL,
                                   coarse ? g->size_mix_scale : 1.0f, corr, !raw && corr->r > 0, 1.0f, 1, accum);
            } else {
                memset(accum, 0, N * sizeof(float));
            }
            float a = isfinite(g->amplitude) ? g->amplitude : 0.0f;
            for (size_t i = 0; i < N; ++i) dens[c][i] = og_san(fmaf(a, accum[i], 0.0f));
        }
    } else {
        int shared_chroma = (debug == FJ_GRAIN_DEBUG_OFF || debug == FJ_GRAIN_DEBUG_DELTA_MIX) && g->chroma_mix < 0.999f &&
                            g->chroma_shared_weight > 0.0f;
        if (shared_chroma) {
            FjVisualGrain sg = *g;
            sg.seed_base ^= 0x7E8A1B9D3F2C65A1ULL;
            sg.seed_base_next ^= 0x7E8A1B9D3F2C65A1ULL;
            o->g = &sg;
            rc = og_mix(&s, dm, 1, shared);
            o->g = g;
        }
        for (int c = 0; c < 3 && !rc; ++c) {
            int independent = g->chroma_independent_weight > 0.0f || !shared_chroma;
            if (independent) rc = og_mix(&s, dens[c], c, accum);
            if (rc) break;
            float sw = og_clamp(g->chroma_shared_weight, 0.0f, 1.0f), iw = og_clamp(g->chroma_independent_weight, 0.0f, 1.0f);
            float amp = g->amplitude;
            float scale = shared_chroma ? 1.0f : amp;
            scale = isfinite(scale) ? scale : 0.0f;
            for (size_t i = 0; i < N; ++i) {
                float d = accum[i];
                if (shared_chroma) {
                    float sv = sw > 0.0f ? shared[i] : 0.0f, iv = iw > 0.0f ? accum[i] : 0.0f;
                    d = og_san(amp * fmaf(sw, sv, iw * iv));
                }
                float mean = debug == FJ_GRAIN_DEBUG_OFF ? dens[c][i] : 0.0f;
                dens[c][i] = og_san(fmaf(scale, d, mean));
            }
        }
    }
    if (!rc && debug != FJ_GRAIN_DEBUG_OFF) {
        float sc = isfinite(g->debug_scale) ? g->debug_scale : 1.0f;
        for (size_t i = 0; i < N; ++i) {
            float a = (dc[i] + dm[i] + dy[i]) * (1.0f / 3.0f);
            if (!isfinite(a)) a = 0.0f;
            dc[i] = dm[i] = dy[i] = fmaf(a, sc, 0.5f);
        }
    }
    free(buf);
    return rc;
}


/* ---------------- scanner post effects (src/Cuda/Scan/JuicerCudaScanPipeline.cu:214-316,
 * :318-446, :586-655, :1944-2037, :2096-2182, :2586-2878) ---------------- */

/* taps of one blur of the record, or radius 0 when that blur is off */
static int post_taps(int radius, float sigma, float** w) {
    *w = NULL;
    if (!(sigma > 0.0f)) return 0;
    if (radius < 1 || radius > 2048 || !isfinite(sigma)) return -1;
    *w = (float*)malloc(sizeof(float) * (size_t)(2 * radius + 1));
    og_taps(radius, sigma, *w);
    return radius;
}

/* separable blur, taps summed in order in FP64; unsharp: plane <- v + a (v - blurred) */
static void post_blur(float* plane, float* tmp, int W, int H, const float* w, int r, int unsharp, float amount) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            double acc = 0.0;
            for (int k = 0; k <= 2 * r; ++k)
                acc += (double)plane[(size_t)y * W + og_reflect_half((long)x - r + k, W)] * (double)w[k];
            tmp[(size_t)y * W + x] = isfinite(acc) ? (float)acc : 0.0f;
        }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            double acc = 0.0;
            for (int k = 0; k <= 2 * r; ++k)
                acc += (double)tmp[(size_t)og_reflect_half((long)y - r + k, H) * W + x] * (double)w[k];
            float blurred = isfinite(acc) ? (float)acc : 0.0f;
            size_t i = (size_t)y * W + x;
            if (unsharp) {
                double v0 = (double)plane[i], o = v0 + (double)amount * (v0 - (double)blurred);
                plane[i] = isfinite(o) ? (float)o : 0.0f;
            } else {
                plane[i] = blurred;
            }
        }
}

/* density planes (C, M, Y) -> print -> scan to linear RGB with glare -> lens blur ->
 * unsharp -> encoded dst. Returns 0, or -1 for a malformed record. */
static float weave_mitchell(const float* plane, int W, int H, float x, float y);
static float gate_bilinear(const float* mask, int W, int H, float x, float y);

int oracle_render_effects(const FjPreparedHostData* h, const FjScannerPostEffects* post, uint64_t seed, int ox,
                          int oy, const FjFilmEffects* fx, const float* dust, const float* mask, const float* dc,
                          const float* dm, const float* dy, const float* src, long src_row_floats, int W, int H,
                          int comps, float* dst, long dst_row_floats, int threads, unsigned* flags_out);

int oracle_render_post(const FjPreparedHostData* h, const FjScannerPostEffects* post, uint64_t seed, int ox, int oy,
                       const float* dc, const float* dm, const float* dy, const float* src, long src_row_floats,
                       int W, int H, int comps, float* dst, long dst_row_floats, int threads, unsigned* flags_out) {
    return oracle_render_effects(h, post, seed, ox, oy, NULL, NULL, NULL, dc, dm, dy, src, src_row_floats, W, H,
                                 comps, dst, dst_row_floats, threads, flags_out);
}

/* Density planes -> (print) -> scan -> post effects -> encoding, with the film defects'
 * output effects (src/Cuda/JuicerCudaExecutor.cpp:1700-1800, :2384-2500): `dust` (or
 * NULL) darkens the print exposure (print route) or the scanned XYZ (direct route);
 * with the gate output on, the weave resamples the linear planes and `mask` (or NULL)
 * multiplies them before encoding (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2096-2182). */
int oracle_render_effects(const FjPreparedHostData* h, const FjScannerPostEffects* post, uint64_t seed, int ox,
                          int oy, const FjFilmEffects* fx, const float* dust, const float* mask, const float* dc,
                          const float* dm, const float* dy, const float* src, long src_row_floats, int W, int H,
                          int comps, float* dst, long dst_row_floats, int threads, unsigned* flags_out) {
    if ((post->flags & ~1u) != 0) return -1;
    const int gate_output = fx && (fx->flags & FJ_EFFECTS_GATE_OUTPUT);
    const int weave = gate_output && (fx->flags & FJ_EFFECTS_WEAVE);
    const float* gate = gate_output && (fx->flags & FJ_EFFECTS_GATE_TRANSMITTANCE) ? mask : NULL;
    Packed pk;
    int rc = pack(h, &pk);
    if (rc) {
        free(pk.lut_store);
        return rc;
    }
    const Pack* p = &pk.p;
    size_t plane = (size_t)W * H;
    float* lin = (float*)malloc(sizeof(float) * plane * 3);
    float* tmp = (float*)malloc(sizeof(float) * plane);
    float* glare = NULL;
    float *gw = NULL, *lw = NULL, *uw = NULL;
    int gr = 0, lr = 0, ur = 0;
    int active = post->hash != 0;
    if (active) {
        lr = post_taps(post->lens_blur_radius, post->lens_blur_sigma_px, &lw);
        ur = post_taps(post->unsharp_radius, post->unsharp_sigma_px, &uw);
        gr = (post->flags & 1u) ? post_taps(post->glare_blur_radius, post->glare_blur_sigma_px, &gw) : 0;
        if (lr < 0 || ur < 0 || gr < 0) {
            free(lin), free(tmp), free(gw), free(lw), free(uw), free(pk.lut_store);
            return -1;
        }
        if (!(isfinite(post->unsharp_amount) && post->unsharp_amount > 0.0f)) ur = 0;
        if (isfinite(post->glare_percent) && post->glare_percent > 0.0f && isfinite(post->glare_roughness)) {
            glare = (float*)malloc(sizeof(float) * plane);
            float mean = fmaxf(0.0f, post->glare_percent), sd = fmaxf(0.0f, post->glare_roughness * post->glare_percent);
            uint32_t medium = p->medium_negative ? 0u : 1u;
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    uint64_t ax = (uint64_t)((int64_t)ox + x), ay = (uint64_t)((int64_t)oy + y);
                    OPhilox ph = {(uint32_t)(seed >> 32), (uint32_t)seed, (uint32_t)ax, (uint32_t)ay, medium, 0};
                    float u1 = fmaf((float)og_philox(&ph), 1.0f / 4294967296.0f, 0.5f / 4294967296.0f);
                    u1 = fminf(fmaxf(u1, 1e-7f), 1.0f);
                    float u2 = fmaf((float)og_philox(&ph), 1.0f / 4294967296.0f, 0.5f / 4294967296.0f);
                    float n = sqrtf(-2.0f * logf(u1)) * cosf(6.28318530717958647692f * u2);
                    float m2 = mean * mean, s2 = sd * sd;
                    float sig2 = logf(1.0f + (s2 / m2));
                    float sig = sqrtf(fmaxf(0.0f, sig2));
                    float mu = logf(fmaxf(1e-12f, mean)) - 0.5f * sig2;
                    float g = expf(mu + sig * n);
                    glare[(size_t)y * W + x] = isfinite(g) ? g : 0.0f;
                }
            if (gr > 0) post_blur(glare, tmp, W, H, gw, gr, 0, 0.0f);
        }
    }
    unsigned flags = 0;
#if defined(_OPENMP)
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads > 0 ? threads : 1) reduction(| : flags)
#endif
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t i = (size_t)y * W + x;
            float D[3] = {dc[i], dm[i], dy[i]};
            if (p->print) print_stage_dust(p, D, dust ? dust[i] : 1.0f);
            double rgb[3];
            if (!scan_lin_dust(p, D, rgb, glare ? glare[i] : -1.0f, dust && !p->print ? dust + i : NULL)) {
                flags |= 1u;
                rgb[0] = rgb[1] = rgb[2] = 0.0;
            }
            for (int c = 0; c < 3; ++c) lin[c * plane + i] = (float)rgb[c];
        }
    for (int c = 0; c < 3 && lr > 0; ++c) post_blur(lin + c * plane, tmp, W, H, lw, lr, 0, 0.0f);
    for (int c = 0; c < 3 && ur > 0; ++c) post_blur(lin + c * plane, tmp, W, H, uw, ur, 1, post->unsharp_amount);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t i = (size_t)y * W + x;
            double rgb[3] = {(double)lin[i], (double)lin[plane + i], (double)lin[2 * plane + i]};
            if (weave) {
                float cx = 0.5f * (float)(W - 1), cy = 0.5f * (float)(H - 1);
                float px = (float)x - cx, py = (float)y - cy;
                float sx = fx->weave_cos_rot * px - fx->weave_sin_rot * py + cx + fx->weave_dx_px;
                float sy = fx->weave_sin_rot * px + fx->weave_cos_rot * py + cy + fx->weave_dy_px;
                for (int c = 0; c < 3; ++c) rgb[c] = (double)weave_mitchell(lin + c * plane, W, H, sx, sy);
            }
            if (gate && fx->gate_width > 0 && fx->gate_height > 0) {
                double t = (double)gate_bilinear(gate, fx->gate_width, fx->gate_height,
                                                 (float)(fx->roi_offset_x + x) * 0.5f - 0.25f,
                                                 (float)(fx->roi_offset_y + y) * 0.5f - 0.25f);
                for (int c = 0; c < 3; ++c) rgb[c] *= t;
            }
            encode_lin(p, rgb);
            float* o = dst + (size_t)y * dst_row_floats + (size_t)x * comps;
            o[0] = (float)rgb[0];
            o[1] = (float)rgb[1];
            o[2] = (float)rgb[2];
            if (comps == 4) o[3] = src ? src[(size_t)y * src_row_floats + (size_t)x * comps + 3] : 1.0f;
        }
    free(lin), free(tmp), free(glare), free(gw), free(lw), free(uw), free(pk.lut_store);
    if (flags_out) *flags_out = flags;
    return 0;
}

/* ---------------- highlight reconstruction (src/Cuda/Film/JuicerCudaHighlightBoost.cu) ---------------- */

typedef struct {
    int disposition;
    float maximum, protection, protection_res, onset, peak, peak_res, range, range_res, shape, shape_res, tail_exp,
        tail_lin, delta, inv_norm;
} OBoost;

static double hb_normexp(double t) {
    if (t >= 0.03125) return (expm1(t) - t) / (t * t);
    return 0.5 + t * (1.0 / 6.0 + t * (1.0 / 24.0 + t * (1.0 / 120.0 + t * (1.0 / 720.0 +
               t * (1.0 / 5040.0 + t * (1.0 / 40320.0 + t * (1.0 / 362880.0 + t / 3628800.0)))))));
}

static float hb_normf(float t, float res) {
    if (t < 0.5f)
        return 0.5f + t * (1.0f / 6.0f + t * (1.0f / 24.0f + t * (1.0f / 120.0f + t * (1.0f / 720.0f +
                   t * (1.0f / 5040.0f + t * (1.0f / 40320.0f + t * (1.0f / 362880.0f + t / 3628800.0f)))))));
    float num = fmaf(expf(t), res, expm1f(t) - t) - res;
    return num / (t * t);
}

static float hb_sample(float s, const OBoost* w) {
    if (s < w->onset) return s;
    if (s == w->maximum) return w->peak;
    float dist = s - w->protection, vp = dist - s;
    float dres = ((s - (dist - vp)) + (-w->protection - vp)) - w->protection_res;
    float q = dist / w->range;
    float corr = (fmaf(-q, w->range, dist) + dres - q * w->range_res) / w->range;
    float fr = q + corr, vc = fr - q;
    float frres = (q - (fr - vc)) + (corr - vc);
    float t = w->shape * fr;
    float tres = fmaf(w->shape, fr, -t) + w->shape * frres + w->shape_res * fr;
    float frsq = fmaf(2.0f * fr, frres, fr * fr);
    float ratio = frsq * (hb_normf(t, tres) * w->inv_norm);
    if (w->shape >= 0.5f && ratio >= 0.5f) {
        float gap = w->maximum - s, gf = gap / w->range;
        float gres = (fmaf(-gf, w->range, gap) - gf * w->range_res) / w->range;
        float d = w->shape * gf;
        float dr = fmaf(w->shape, gf, -d) + w->shape * gres + w->shape_res * gf;
        float ome = fmaf(expf(-d), dr, -expm1f(-d));
        float tail = fmaf(ome, w->tail_exp, -(d + dr) * w->tail_lin);
        float ep = w->peak - gap, vg = w->peak - ep;
        float epres = (w->peak - (ep + vg)) + (vg - gap);
        return ep + ((epres + w->peak_res) - w->delta * tail);
    }
    return s + w->delta * ratio;
}

/* carrier planes B, G, R boosted in place; returns the disposition (0 bypass, 1 applied,
 * 2 invalid carrier, 3 peak overflow) */
int oracle_highlight_boost(uint64_t recipe_hash, double protection, double sharpness, double peak_gain, float* b,
                           float* g, float* r, long stride, int W, int H) {
    if (recipe_hash == 0 || W <= 0 || H <= 0) return 0;
    float mx = 0.0f;
    int invalid = 0;
    float* planes[3] = {r, g, b};
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < 3; ++c) {
                float v = planes[c][(size_t)y * stride + x];
                if (isfinite(v) && v >= 0.0f) mx = fmaxf(mx, v);
                else invalid = 1;
            }
    OBoost w;
    memset(&w, 0, sizeof(w));
    double maximum = mx;
    w.maximum = mx;
    if (invalid) return 2;
    if (maximum <= protection) return 0;
    double peak = maximum * peak_gain;
    if (peak > (double)FLT_MAX) return 3;
    double range = maximum - protection;
    double shape = sharpness * range / maximum;
    double norm = hb_normexp(shape);
    w.protection = (float)protection;
    w.protection_res = (float)(protection - (double)w.protection);
    w.onset = (double)w.protection <= protection ? nextafterf(w.protection, INFINITY) : w.protection;
    w.peak = (float)peak;
    w.peak_res = (float)(peak - (double)w.peak);
    w.range = (float)range;
    w.range_res = (float)(range - (double)w.range);
    w.shape = (float)shape;
    w.shape_res = (float)(shape - (double)w.shape);
    if (w.shape >= 0.5f) {
        double den = shape * shape * norm;
        w.tail_exp = (float)(exp(shape) / den);
        w.tail_lin = (float)(1.0 / den);
    }
    w.delta = (float)(maximum * (peak_gain - 1.0));
    w.inv_norm = (float)(1.0 / norm);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < 3; ++c) {
                float* v = &planes[c][(size_t)y * stride + x];
                *v = hb_sample(*v, &w);
            }
    return 1;
}

/* ---------------- film and gate defects (src/Cuda/Scan/JuicerCudaScanPipeline.cu:801-1360, :2056-2094) ---------------- */

static float weave_mitchell(const float* plane, int W, int H, float x, float y) {
    x = fminf(fmaxf(x, 0.0f), (float)(W - 1));
    y = fminf(fmaxf(y, 0.0f), (float)(H - 1));
    int ix = (int)floorf(x), iy = (int)floorf(y);
    float tx = x - (float)ix, ty = y - (float)iy;
    float wx[4] = {mitchell(tx + 1.0f), mitchell(tx), mitchell(tx - 1.0f), mitchell(tx - 2.0f)};
    float wy[4] = {mitchell(ty + 1.0f), mitchell(ty), mitchell(ty - 1.0f), mitchell(ty - 2.0f)};
    double acc = 0.0;
    for (int j = 0; j < 4; ++j) {
        int sy = iy + j - 1;
        sy = sy < 0 ? 0 : sy > H - 1 ? H - 1 : sy;
        for (int i = 0; i < 4; ++i) {
            int sx = ix + i - 1;
            sx = sx < 0 ? 0 : sx > W - 1 ? W - 1 : sx;
            acc += (double)wy[j] * wx[i] * (double)plane[(size_t)sy * W + sx];
        }
    }
    return (float)acc;
}

static float gate_bilinear(const float* m, int W, int H, float x, float y) {
    float fx = fminf(fmaxf(x, 0.0f), (float)(W - 1)), fy = fminf(fmaxf(y, 0.0f), (float)(H - 1));
    int x0 = (int)floorf(fx), y0 = (int)floorf(fy);
    int x1 = x0 + 1 < W ? x0 + 1 : x0, y1 = y0 + 1 < H ? y0 + 1 : y0;
    float tx = fx - (float)x0, ty = fy - (float)y0;
    float m0 = m[y0 * W + x0] + (m[y0 * W + x1] - m[y0 * W + x0]) * tx;
    float m1 = m[y1 * W + x0] + (m[y1 * W + x1] - m[y1 * W + x0]) * tx;
    return m0 + (m1 - m0) * ty;
}

static uint64_t od_mix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

static float od_lane(uint64_t id, unsigned k) {
    uint64_t h = od_mix(id ^ (0xD6E8FEB86659FD93ULL * ((uint64_t)k + 1ULL)));
    return (float)((h >> 40) & 0xFFFFFFu) * (1.0f / 16777216.0f);
}

typedef struct {
    float cx, cy, xmin, xmax, ymin, ymax, strength, softness;
    float ex[3], ey[3], ea[3], eb[3], ec[3];
    float px[4], py[4], w[4], d[4];
    int stroke, active;
} OParticle;

static float od_mixture(float u, float v, float lo, float bulk, float hi, float tail) {
    float t = v * v * v;
    return u < tail ? bulk + (hi - bulk) * t : lo + (bulk - lo) * t;
}

static void od_stroke(OParticle* q, uint64_t h, float length, float drift, float angle, const float* t,
                      const float* w, const float* d) {
    float dx[4] = {0.0f, (od_lane(h, 12) - 0.5f) * drift * length, (od_lane(h, 13) - 0.5f) * drift * length,
                   (od_lane(h, 14) - 0.5f) * drift * length};
    float total = 0.0f, widest = 0.0f;
    for (int i = 1; i < 4; ++i) total += hypotf(dx[i] - dx[i - 1], length * (t[i] - t[i - 1]));
    for (int i = 0; i < 4; ++i) widest = fmaxf(widest, w[i]);
    float norm = length / total, c = cosf(angle), s = sinf(angle);
    q->stroke = 1;
    q->xmin = q->ymin = 1.0e30f;
    q->xmax = q->ymax = -1.0e30f;
    for (int i = 0; i < 4; ++i) {
        float yy = (t[i] - 0.5f) * length * norm, xx = dx[i] * norm;
        q->px[i] = xx * c - yy * s;
        q->py[i] = xx * s + yy * c;
        q->w[i] = w[i];
        q->d[i] = d[i];
        q->xmin = fminf(q->xmin, q->px[i] - widest * 0.5f);
        q->xmax = fmaxf(q->xmax, q->px[i] + widest * 0.5f);
        q->ymin = fminf(q->ymin, q->py[i] - widest * 0.5f);
        q->ymax = fmaxf(q->ymax, q->py[i] + widest * 0.5f);
    }
}

static float od_opacity(const FjDust* d, int fiber, float u) {
    float lo = fiber ? d->fiber_opacity_min : d->compact_opacity_min;
    float f = fiber ? d->fiber_opacity_faint_end : d->compact_opacity_faint_end;
    float m = fiber ? d->fiber_opacity_intermediate_end : d->compact_opacity_intermediate_end;
    float hi = fiber ? d->fiber_opacity_max : d->compact_opacity_max;
    float c1 = d->opacity_faint_cumulative, c2 = d->opacity_intermediate_cumulative;
    if (u < c1) return lo + (f - lo) * (u / c1);
    if (u < c2) return f + (m - f) * ((u - c1) / (c2 - c1));
    return m + (hi - m) * ((u - c2) / (1.0f - c2));
}

static OParticle od_particle(const FjFilmEffects* e, int fam, int64_t cxl, int64_t cyl, int slot, int offx, int offy) {
    OParticle q;
    memset(&q, 0, sizeof(q));
    const FjDust* du = fam == 0 ? &e->film_dust : &e->gate_dust;
    const FjScratch* sc = fam == 1 ? &e->film_scratch : &e->gate_scratch;
    int dust = fam == 0 || fam == 2;
    uint64_t h = od_mix(e->session_seed);
    if (fam < 2) h = od_mix(h ^ od_mix(e->clip_token));
    h = od_mix(h ^ (uint64_t)cxl);
    h = od_mix(h ^ (uint64_t)cyl);
    h = od_mix(h ^ (0x8EBC6AF09C88C6E3ULL * (uint64_t)(fam + 1)));
    h = od_mix(h ^ (uint64_t)slot);
    if (od_lane(h, 0) >= (dust ? du->slot_probability : sc->slot_probability)) return q;
    q.cx = ((float)offx + od_lane(h, 1)) * (dust ? du->cell_width_mm : sc->cell_width_mm);
    q.cy = ((float)offy + od_lane(h, 2)) * (dust ? du->cell_height_mm : sc->cell_height_mm);
    q.active = 1;
    if (dust) {
        float angle = od_lane(h, 4) * 6.28318530718f;
        int fiber = od_lane(h, 5) < du->fiber_fraction;
        q.strength = od_opacity(du, fiber, od_lane(h, 3));
        if (fiber) {
            float len = du->fiber_length_min_mm + (du->fiber_length_max_mm - du->fiber_length_min_mm) * od_lane(h, 6);
            float wid = du->fiber_width_min_mm + (du->fiber_width_max_mm - du->fiber_width_min_mm) * od_lane(h, 7);
            float u = od_lane(h, 47);
            q.softness = fminf(du->softness_min_mm + (du->softness_max_mm - du->softness_min_mm) * u * u,
                               wid * du->softness_size_cap_fraction);
            float t[4] = {0.0f,
                          du->fiber_first_knot_min + (du->fiber_first_knot_max - du->fiber_first_knot_min) * od_lane(h, 30),
                          du->fiber_second_knot_min +
                              (du->fiber_second_knot_max - du->fiber_second_knot_min) * od_lane(h, 31),
                          1.0f};
            float span = du->fiber_interior_width_max_fraction - du->fiber_interior_width_min_fraction;
            float w[4] = {0.0f, wid * (du->fiber_interior_width_min_fraction + span * od_lane(h, 21)),
                          wid * (du->fiber_interior_width_min_fraction + span * od_lane(h, 22)), 0.0f};
            float d[4] = {1.0f, 1.0f, 1.0f, 1.0f};
            od_stroke(&q, h, len, du->fiber_drift_fraction, angle, t, w, d);
        } else {
            float dia = od_mixture(od_lane(h, 6), od_lane(h, 7), du->diameter_min_mm, du->diameter_bulk_max_mm,
                                   du->diameter_max_mm, du->diameter_tail_fraction);
            float u = od_lane(h, 47);
            q.softness = fminf(du->softness_min_mm + (du->softness_max_mm - du->softness_min_mm) * u * u,
                               dia * du->softness_size_cap_fraction);
            float ox[3] = {0}, oy[3] = {0}, rx[3] = {0}, ry[3] = {0}, rot[3] = {0};
            rx[0] = 1.0f;
            ry[0] = du->compact_dominant_aspect_min +
                    (du->compact_dominant_aspect_max - du->compact_dominant_aspect_min) * od_lane(h, 32);
            rot[0] = angle;
            float dc = cosf(angle), ds = sinf(angle), enc = 1.0f;
            for (int i = 1; i < 3; ++i) {
                rx[i] = du->compact_subsidiary_scale_min +
                        (du->compact_subsidiary_scale_max - du->compact_subsidiary_scale_min) * od_lane(h, 32 + i * 5);
                float asp = du->compact_subsidiary_aspect_min +
                            (du->compact_subsidiary_aspect_max - du->compact_subsidiary_aspect_min) * od_lane(h, 33 + i * 5);
                ry[i] = rx[i] * asp;
                float polar = od_lane(h, 34 + i * 5) * 6.28318530718f;
                float radial = du->compact_subsidiary_offset_max * sqrtf(od_lane(h, 35 + i * 5));
                float lx = radial * cosf(polar), ly = radial * ry[0] * sinf(polar);
                ox[i] = lx * dc - ly * ds;
                oy[i] = lx * ds + ly * dc;
                rot[i] = angle + (2.0f * od_lane(h, 36 + i * 5) - 1.0f) * du->compact_subsidiary_angle_max_radians;
                enc = fmaxf(enc, hypotf(ox[i], oy[i]) + fmaxf(rx[i], ry[i]));
            }
            float scale = dia * 0.5f / enc;
            q.xmin = q.ymin = 1.0e30f;
            q.xmax = q.ymax = -1.0e30f;
            for (int i = 0; i < 3; ++i) {
                float a = rx[i] * scale, b = ry[i] * scale, c = cosf(rot[i]), s = sinf(rot[i]);
                q.ex[i] = ox[i] * scale;
                q.ey[i] = oy[i] * scale;
                q.ea[i] = c * c / (a * a) + s * s / (b * b);
                q.eb[i] = c * s * (1.0f / (a * a) - 1.0f / (b * b));
                q.ec[i] = s * s / (a * a) + c * c / (b * b);
                float hx = sqrtf(a * a * c * c + b * b * s * s), hy = sqrtf(a * a * s * s + b * b * c * c);
                q.xmin = fminf(q.xmin, q.ex[i] - hx);
                q.xmax = fmaxf(q.xmax, q.ex[i] + hx);
                q.ymin = fminf(q.ymin, q.ey[i] - hy);
                q.ymax = fmaxf(q.ymax, q.ey[i] + hy);
            }
        }
    } else {
        q.strength = sc->strength_min + (sc->strength_max - sc->strength_min) * od_lane(h, 3);
        float len = od_mixture(od_lane(h, 6), od_lane(h, 7), sc->length_min_mm, sc->length_bulk_max_mm,
                               sc->length_max_mm, sc->length_tail_fraction);
        float wid = od_mixture(od_lane(h, 8), od_lane(h, 9), sc->width_min_mm, sc->width_bulk_max_mm, sc->width_max_mm,
                               sc->width_tail_fraction);
        float u = od_lane(h, 47);
        q.softness = fminf(sc->softness_min_mm + (sc->softness_max_mm - sc->softness_min_mm) * u * u,
                           wid * sc->softness_size_cap_fraction);
        float t[4] = {0.0f, 0.0f, 0.0f, 1.0f}, w[4], d[4], angle = 0.0f;
        int gap = od_lane(h, 30) < sc->interruption_probability;
        if (gap) {
            float c = sc->gap_center_min + (sc->gap_center_max - sc->gap_center_min) * od_lane(h, 31);
            float sp = sc->gap_span_min + (sc->gap_span_max - sc->gap_span_min) * od_lane(h, 32);
            t[1] = c - sp * 0.5f;
            t[2] = c + sp * 0.5f;
        } else {
            t[1] = sc->first_knot_min + (sc->first_knot_max - sc->first_knot_min) * od_lane(h, 31);
            t[2] = sc->second_knot_min + (sc->second_knot_max - sc->second_knot_min) * od_lane(h, 32);
        }
        for (int i = 0; i < 4; ++i) {
            float wf = sc->interior_width_min_fraction +
                       (sc->interior_width_max_fraction - sc->interior_width_min_fraction) * od_lane(h, 33 + i);
            w[i] = (i == 1 || i == 2 || od_lane(h, 37 + i) < sc->endpoint_abrupt_probability) ? wid * wf : 0.0f;
            d[i] = sc->interior_depth_min_fraction +
                   (sc->interior_depth_max_fraction - sc->interior_depth_min_fraction) * od_lane(h, 41 + i);
        }
        if (gap) d[1] = d[2] = 0.0f;
        if (len <= sc->scuff_length_max_mm && od_lane(h, 45) < sc->scuff_probability)
            angle = (2.0f * od_lane(h, 46) - 1.0f) * sc->scuff_angle_max_radians;
        od_stroke(&q, h, len, sc->drift_fraction, angle, t, w, d);
    }
    return q;
}

static float od_section(const OParticle* q, float y, float bx, float by) {
    float lo[5] = {0}, hi[5] = {0}, dep[5] = {0};
    int n = 0;
    for (int i = 0; i < 3; ++i) {
        float a = 0.0f, b = 0.0f;
        if (!q->stroke) {
            float dy = y - q->ey[i];
            float disc = q->ea[i] - (q->ea[i] * q->ec[i] - q->eb[i] * q->eb[i]) * dy * dy;
            if (disc <= 0.0f) continue;
            float c = q->ex[i] - q->eb[i] * dy / q->ea[i], r = sqrtf(disc) / q->ea[i];
            a = c - r;
            b = c + r;
        } else {
            float dx = q->px[i + 1] - q->px[i], dy = q->py[i + 1] - q->py[i];
            float inv = 1.0f / sqrtf(dx * dx + dy * dy);
            float nx = -dy * inv * 0.5f, ny = dx * inv * 0.5f;
            float vx[4] = {q->px[i] + nx * q->w[i], q->px[i + 1] + nx * q->w[i + 1], q->px[i + 1] - nx * q->w[i + 1],
                           q->px[i] - nx * q->w[i]};
            float vy[4] = {q->py[i] + ny * q->w[i], q->py[i + 1] + ny * q->w[i + 1], q->py[i + 1] - ny * q->w[i + 1],
                           q->py[i] - ny * q->w[i]};
            a = 1.0e30f;
            b = -1.0e30f;
            for (int k = 0; k < 4; ++k) {
                int k1 = (k + 1) % 4;
                if (y >= fminf(vy[k], vy[k1]) && y < fmaxf(vy[k], vy[k1])) {
                    float x = vx[k] + (y - vy[k]) / (vy[k1] - vy[k]) * (vx[k1] - vx[k]);
                    a = fminf(a, x);
                    b = fmaxf(b, x);
                }
            }
        }
        a = fmaxf(bx, a);
        b = fminf(by, b);
        if (b > a) {
            dep[n] = 1.0f;
            if (q->stroke) {
                float dx = q->px[i + 1] - q->px[i], dy = q->py[i + 1] - q->py[i];
                float mid = 0.5f * (a + b), den = dx * dx + dy * dy;
                float t = fminf(1.0f, fmaxf(0.0f, ((mid - q->px[i]) * dx + (y - q->py[i]) * dy) / den));
                dep[n] = q->d[i] + (q->d[i + 1] - q->d[i]) * t;
            }
            lo[n] = a;
            hi[n] = b;
            ++n;
        }
    }
    if (q->stroke)
        for (int i = 1; i < 3; ++i) {
            float r = q->w[i] * 0.5f, dy = y - q->py[i];
            if (fabsf(dy) >= r) continue;
            float ch = sqrtf(fmaxf(0.0f, r * r - dy * dy));
            float a = fmaxf(bx, q->px[i] - ch), b = fminf(by, q->px[i] + ch);
            if (b > a) {
                lo[n] = a;
                hi[n] = b;
                dep[n] = q->d[i];
                ++n;
            }
        }
    float ends[10] = {0};
    for (int i = 0; i < n; ++i) {
        ends[2 * i] = lo[i];
        ends[2 * i + 1] = hi[i];
    }
    for (int i = 1; i < 2 * n; ++i)
        for (int j = i; j > 0 && ends[j] < ends[j - 1]; --j) {
            float v = ends[j];
            ends[j] = ends[j - 1];
            ends[j - 1] = v;
        }
    float len = 0.0f;
    for (int i = 1; i < 2 * n; ++i) {
        float mid = (ends[i - 1] + ends[i]) * 0.5f, st = 0.0f;
        for (int k = 0; k < n; ++k)
            if (mid >= lo[k] && mid <= hi[k]) st = fmaxf(st, dep[k]);
        len += (ends[i] - ends[i - 1]) * st;
    }
    return len;
}

static float od_coverage(const OParticle* q, float x, float y, float sx, float sy) {
    x -= q->cx;
    y -= q->cy;
    if (x + sx * 0.5f + q->softness < q->xmin || x - sx * 0.5f - q->softness > q->xmax ||
        y + sy * 0.5f + q->softness < q->ymin || y - sy * 0.5f - q->softness > q->ymax)
        return 0.0f;
    float area = 0.0f;
    for (int soft = 0; soft < 3; ++soft) {
        float shift = ((float)soft - 1.0f) * q->softness;
        float bottom = fmaxf(q->ymin, y - sy * 0.5f + shift), top = fminf(q->ymax, y + sy * 0.5f + shift);
        if (!(top > bottom)) continue;
        float sum = 0.0f;
        for (int row = 0; row < 8; ++row) {
            float yy = bottom + ((float)row + 0.5f) * (top - bottom) / 8.0f;
            for (int col = 0; col < 3; ++col) {
                float off = ((float)col - 1.0f) * q->softness;
                sum += od_section(q, yy, x - sx * 0.5f + off, x + sx * 0.5f + off);
            }
        }
        area += sum * (top - bottom) / 72.0f;
    }
    return fminf(1.0f, fmaxf(0.0f, area / (sx * sy)));
}

/* Retained fraction of one family over a W x H pixel grid whose first pixel is (gx0, gy0)
 * in the family's frame; candidates per 32 x 8 tile as the reference enumerates them. */
static void od_family(const FjFilmEffects* e, int fam, int gx0, int gy0, int W, int H, float scale, float* out) {
    int dust = fam == 0 || fam == 2;
    const FjDust* dp = fam == 0 ? &e->film_dust : &e->gate_dust;
    const FjScratch* sp = fam == 1 ? &e->film_scratch : &e->gate_scratch;
    for (size_t i = 0; i < (size_t)W * H; ++i) out[i] = 1.0f;
    if (!((dust ? dp->slot_probability : sp->slot_probability) > 0.0f)) return;
    float cw = dust ? dp->cell_width_mm : sp->cell_width_mm, ch = dust ? dp->cell_height_mm : sp->cell_height_mm;
    float sux = dust ? dp->support_x_mm + dp->softness_max_mm : sp->support_x_mm + sp->softness_max_mm;
    float suy = dust ? dp->support_y_mm + dp->softness_max_mm : sp->support_y_mm + sp->softness_max_mm;
    const FjDefectOrigin* o = &e->origins[fam];
    float stx = e->sample_step_x_mm * scale, sty = e->sample_step_y_mm * scale;
    float bx = o->local_x_mm, by = o->local_y_mm;
    for (int ty = 0; ty < H; ty += 8)
        for (int tx = 0; tx < W; tx += 32) {
            int tfx = gx0 + tx, tfy = gy0 + ty;
            int x0 = (int)floorf((bx + (float)tfx * stx - sux) / cw), y0 = (int)floorf((by + (float)tfy * sty - suy) / ch);
            int x1 = (int)floorf((bx + (float)(tfx + 32) * stx + sux) / cw);
            int y1 = (int)floorf((by + (float)(tfy + 8) * sty + suy) / ch);
            int cols = x1 - x0 + 1, total = cols * (y1 - y0 + 1) * 2;
            for (int ord = 0; ord < total; ++ord) {
                int dx = x0 + (ord / 2) % cols, dy = y0 + (ord / 2) / cols;
                OParticle q = od_particle(e, fam, o->cell_x + dx, o->cell_y + dy, ord % 2, dx, dy);
                if (!q.active) continue;
                for (int yy = ty; yy < ty + 8 && yy < H; ++yy)
                    for (int xx = tx; xx < tx + 32 && xx < W; ++xx) {
                        float px = bx + ((float)(gx0 + xx) + 0.5f) * stx, py = by + ((float)(gy0 + yy) + 0.5f) * sty;
                        out[(size_t)yy * W + xx] *= 1.0f - q.strength * od_coverage(&q, px, py, stx, sty);
                    }
            }
        }
}

/* film dust -> `dust` (when on), film scratches scale C, M, Y (when on) */
int oracle_film_defects(const FjFilmEffects* e, int W, int H, float* c, float* m, float* y, float* dust) {
    float* ret = (float*)malloc(sizeof(float) * (size_t)W * H);
    if (!ret) return 2;
    if (e->film_dust.slot_probability > 0.0f && dust)
        od_family(e, 0, e->roi_offset_x, e->roi_offset_y, W, H, 1.0f, dust);
    if (e->film_scratch.slot_probability > 0.0f) {
        od_family(e, 1, e->roi_offset_x, e->roi_offset_y, W, H, 1.0f, ret);
        for (size_t i = 0; i < (size_t)W * H; ++i) {
            c[i] *= ret[i];
            m[i] *= ret[i];
            y[i] *= ret[i];
        }
    }
    free(ret);
    return 0;
}

/* gate dust x gate scratch at the gate grid */
int oracle_gate_mask(const FjFilmEffects* e, float* mask, int W, int H) {
    float* s = (float*)malloc(sizeof(float) * (size_t)W * H);
    if (!s) return 2;
    od_family(e, 2, 0, 0, W, H, 2.0f, mask);
    od_family(e, 3, 0, 0, W, H, 2.0f, s);
    for (size_t i = 0; i < (size_t)W * H; ++i) mask[i] *= s[i];
    free(s);
    return 0;
}

/* ---------------- tables of the parameter-fitting chain ----------------
 * The packed tables (as the render packs them) that an FP64 transcription of the
 * per-pixel chain needs: capture curves on the shared log-exposure axis and the DIR
 * compensated axes (B, G, R), the DIR matrix, reference densities and donor knees in
 * the same index space, the print's spectral tables and curves, the scan bounds,
 * correction and colour matrices. The scanner LUT is the one oracle_scanner_lut builds
 * from the same record. Returns 0, or 1 when a curve holds more than
 * ORACLE_FIT_MAX_SAMPLES samples, 2 when packing fails. */
#define ORACLE_FIT_MAX_SAMPLES 1024
typedef struct {
    int32_t n, dir_mode, print, np, medium_negative, res, corr_active, pad;
    float log_exposure[ORACLE_FIT_MAX_SAMPLES];
    float density_bgr[3][ORACLE_FIT_MAX_SAMPLES];
    float axes_bgr[3][ORACLE_FIT_MAX_SAMPLES];
    float gamma_bgr[3], dir_m[9], dir_dref[3], dir_k[3];
    float eps_cmy[NL * 3], base[NL], illuminant[NL], sens_cmy[NL * 3];
    float midgray, preflash, preflash_raw[3], print_exposure, print_route;
    float print_log_exposure[ORACLE_FIT_MAX_SAMPLES];
    float print_density_cmy[3][ORACLE_FIT_MAX_SAMPLES];
    float min_cmy[3], inv_cmy[3], corr_slope, corr_offset, cat02[9], xyz_to_rgb[9];
    float dir_dmax[3], dir_rcref[3], dir_rkr[3]; /* positive stocks: donors and receivers */
} OracleFitTables;

int oracle_fit_tables(const FjPreparedHostData* h, OracleFitTables* t) {
    Packed pk;
    memset(t, 0, sizeof(*t));
    if (pack(h, &pk)) {
        free(pk.lut_store);
        return 2;
    }
    const Pack* p = &pk.p;
    free(pk.lut_store);
    const int n = p->dens[0].n;
    if (n > ORACLE_FIT_MAX_SAMPLES) return 1;
    t->n = n;
    t->dir_mode = p->dir_mode;
    t->print = p->print;
    t->medium_negative = p->medium_negative;
    t->res = p->res;
    t->corr_active = p->corr_active;
    for (int i = 0; i < n; ++i) t->log_exposure[i] = p->dens[0].x[i];
    for (int c = 0; c < 3; ++c) {
        t->gamma_bgr[c] = p->gamma_bgr[c];
        for (int i = 0; i < n; ++i) t->density_bgr[c][i] = p->dens[c].y[(size_t)i * p->dens[c].ystride];
        if (p->dir_mode != FJ_DIR_INACTIVE)
            for (int i = 0; i < n; ++i) t->axes_bgr[c][i] = p->dirc[c].x[i];
        t->dir_dref[c] = p->dref[c];
        t->dir_k[c] = p->dk[c];
        t->dir_dmax[c] = p->dmax[c];
        t->dir_rcref[c] = p->rcref[c];
        t->dir_rkr[c] = p->rkr[c];
        t->min_cmy[c] = p->min_cmy[c];
        t->inv_cmy[c] = p->inv_cmy[c];
    }
    memcpy(t->dir_m, p->M, sizeof(t->dir_m));
    if (p->print) {
        const int np = p->pdc[0].n;
        if (np > ORACLE_FIT_MAX_SAMPLES) return 1;
        t->np = np;
        for (int i = 0; i < np; ++i) t->print_log_exposure[i] = p->pdc[0].x[i];
        for (int c = 0; c < 3; ++c)
            for (int i = 0; i < np; ++i) t->print_density_cmy[c][i] = p->pdc[c].y[(size_t)i * p->pdc[c].ystride];
        memcpy(t->eps_cmy, p->eps_c_src, sizeof(t->eps_cmy));
        memcpy(t->base, p->base_src, sizeof(t->base));
        memcpy(t->illuminant, p->pillum, sizeof(t->illuminant));
        memcpy(t->sens_cmy, p->psens, sizeof(t->sens_cmy));
        t->midgray = p->midgray;
        t->preflash = p->preflash;
        memcpy(t->preflash_raw, p->preflash_raw, sizeof(t->preflash_raw));
        t->print_exposure = p->print_exposure;
        t->print_route = p->print_route;
    }
    t->corr_slope = p->corr_slope;
    t->corr_offset = p->corr_offset;
    memcpy(t->cat02, p->cat02, sizeof(t->cat02));
    memcpy(t->xyz_to_rgb, p->xyz_rgb, sizeof(t->xyz_to_rgb));
    return 0;
}
