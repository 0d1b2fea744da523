// fjb_recipe.cpp -- FjPreparedHostData -> device-resident recipe tables + kernel params.
//
// The decode follows the reference's packing rules so that the kernels see the same
// numbers the reference kernels see:
//  - film payload: src/Cuda/JuicerCudaFilmPayloads.cpp:28-197 (BGR order, gamma
//    factors, DIR matrix transpose into [donor BGR][receiver BGR], exp2 of manual EV);
//  - curves: src/Cuda/JuicerCudaResources.cpp:1379-1393 (domain [0, n-1]), :3838-3840
//    (compensated DIR axes paired with the normal density ordinates);
//  - print payload: src/Cuda/JuicerCudaResources.cpp:4186-4254, :4335-4420 (route
//    correction of the print stage = scanner correction exposure scale,
//    src/Cuda/JuicerCudaExecutor.cpp:2938-2944);
//  - scan range: src/Cuda/JuicerCudaResources.cpp:3910-3922 (direct routes negate the
//    density minimum);
//  - output colour: native/juicer_cuda_descriptors.cpp:569-601 and
//    src/Cuda/JuicerCudaExecutor.cpp:962-1011, :1590-1607.
// The layout is this project's: curves concatenated into one blob staged to shared
// memory, print spectra folded and stored as kernel parameters, TC LUT and scanner
// nodes as float4 vectors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "fjb_internal.h"
#include "fjb_recipe.h"

namespace fjb {

namespace {

bool span_ok(const FjFloatSpan& s, size_t count) { return s.data != nullptr && s.count == count; }

template <typename T>
cudaError_t upload(T** dst, const void* src, size_t bytes, cudaStream_t stream) {
    *dst = nullptr;
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), bytes);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream);
}

// Enables the uniform-grid interval guess for a curve whose abscissa is strictly
// increasing with every step within 25 % of the mean step (then the guessed cell is
// at most one off and two correction steps always land on the exact interval).
void set_curve_guess(const std::vector<float>& blob, CurveRef& c) {
    c.guess = 0;
    if (c.n < 2) return;
    const float* x = blob.data() + c.x;
    const double span = (double)x[c.n - 1] - (double)x[0];
    if (!(span > 0.0) || !std::isfinite(span)) return;
    const double mean = span / (c.n - 1);
    for (int i = 0; i + 1 < c.n; ++i) {
        const double d = (double)x[i + 1] - (double)x[i];
        if (!(d > 0.0) || std::fabs(d - mean) > 0.25 * mean) return;
    }
    c.x0 = x[0];
    c.inv_dx = (float)((c.n - 1) / span);
    c.guess = 1;
}

} // namespace

cudaError_t Recipe::ensure_tc_raw(size_t pixels) noexcept {
    const size_t need = 3 * pixels;
    if (tc_raw && tc_raw_floats >= need) return cudaSuccess;
    if (tc_raw) cudaFree(tc_raw);
    tc_raw = nullptr;
    tc_raw_floats = 0;
    void* ptr = nullptr;
    cudaError_t e = cudaMalloc(&ptr, need * sizeof(float));
    if (e != cudaSuccess) return e;
    tc_raw = static_cast<float*>(ptr);
    tc_raw_floats = need;
    return cudaSuccess;
}

void Recipe::release() noexcept {
    void* ptrs[] = {curves, tc_lut, mallett_basis, mallett_illum, film_sens_bgr, gamut_cmax, flags,
                    lut.nodes, lut.log2_xyz, lut.slope_c, lut.slope_m, lut.slope_y, lut.cell_min, lut.cell_max,
                    lut.packed_nodes, lut.packed_cells, lut.failure, lut_spectra, meter_scratch, layer_curves,
                    tc_raw};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    curves = nullptr;
    tc_lut = nullptr;
    mallett_basis = mallett_illum = film_sens_bgr = gamut_cmax = nullptr;
    flags = nullptr;
    lut = ScannerLutDevice{};
    lut_spectra = nullptr;
    meter_scratch = nullptr;
    layer_curves = nullptr;
    tc_raw = nullptr;
    tc_raw_floats = 0;
    layer_n = 0;
}

cudaError_t alloc_scanner_lut(int r, ScannerLutDevice& lut) {
    const size_t nodes = (size_t)r * r * r * 3;
    const size_t cells = (size_t)(r - 1) * (r - 1) * (r - 1) * 3;
    cudaError_t e;
    if ((e = cudaMalloc(&lut.nodes, nodes * sizeof(double))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.log2_xyz, nodes * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.slope_c, nodes * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.slope_m, nodes * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.slope_y, nodes * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.cell_min, cells * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.cell_max, cells * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.packed_nodes, nodes * sizeof(float4))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.packed_cells, (cells / 3) * 2 * sizeof(float4))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&lut.failure, sizeof(unsigned))) != cudaSuccess) return e;
    return cudaSuccess;
}

void free_scanner_lut(ScannerLutDevice& lut) {
    void* ptrs[] = {lut.nodes, lut.log2_xyz, lut.slope_c, lut.slope_m, lut.slope_y, lut.cell_min,
                    lut.cell_max, lut.packed_nodes, lut.packed_cells, lut.failure};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    lut = ScannerLutDevice{};
}

// Uploads the scanner spectra (as FP64) and builds the PCHIP LUT on `stream`.
// `doubles` receives the device allocation holding the seven spectra.
cudaError_t build_scanner_lut(const LutSource& src, ScannerLutDevice& lut, double** doubles, cudaStream_t stream) {
    const int k = src.k;
    std::vector<double> host((size_t)7 * k, 0.0);
    for (int i = 0; i < k; ++i) {
        host[0 * k + i] = src.eps_c[i];
        host[1 * k + i] = src.eps_m[i];
        host[2 * k + i] = src.eps_y[i];
        host[3 * k + i] = src.wx[i];
        host[4 * k + i] = src.wy[i];
        host[5 * k + i] = src.wz[i];
        host[6 * k + i] = src.baseline ? src.baseline[i] : 0.0;
    }
    cudaError_t e = cudaMalloc(doubles, host.size() * sizeof(double));
    if (e != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(*doubles, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, stream)) !=
        cudaSuccess)
        return e;
    if ((e = alloc_scanner_lut(src.resolution, lut)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(lut.failure, 0, sizeof(unsigned), stream)) != cudaSuccess) return e;
    ScannerLutSpec spec{};
    spec.eps_c = *doubles;
    spec.eps_m = *doubles + k;
    spec.eps_y = *doubles + 2 * k;
    spec.wx = *doubles + 3 * k;
    spec.wy = *doubles + 4 * k;
    spec.wz = *doubles + 5 * k;
    spec.baseline = src.baseline ? *doubles + 6 * k : nullptr;
    spec.k = k;
    spec.inv_yn = (double)src.inv_yn;
    for (int c = 0; c < 3; ++c) {
        spec.range_min_cmy[c] = src.range_min_cmy[c];
        spec.inverse_span_cmy[c] = src.inverse_span_cmy[c];
    }
    spec.medium = src.medium;
    spec.resolution = src.resolution;
    e = launch_scanner_lut_build(spec, lut, stream);
    if (e != cudaSuccess) return e;
    // the host staging vector must outlive the async copy
    return cudaStreamSynchronize(stream);
}

bool create_recipe(const FjPreparedHostData& h, cudaStream_t stream, Recipe& r, std::string& why, FjStatus& status) {
    status = FjStatus{FJ_STATUS_PREPARATION_FAILURE, FJ_API_NONE, 0};
    r = Recipe{};
    PixelParams& p = r.params;
    std::memset(&p, 0, sizeof(p));
    if (h.route > FJ_ROUTE_POSITIVE_PRINT) {
        why = "unsupported route";
        status.category = FJ_STATUS_UNSUPPORTED_INPUT;
        return false;
    }
    const bool print = h.route == FJ_ROUTE_NEGATIVE_PRINT || h.route == FJ_ROUTE_POSITIVE_PRINT;
    p.route = print ? kRoutePrint : kRouteDirect;
    r.print = print;
    r.positive_film = h.capture_polarity == FJ_POLARITY_POSITIVE;

    // ---- exposure ----
    const FjFilmExposure& ex = h.film_exposure;
    if (ex.method > FJ_RAW_ARCTIC_2026_BETA04) {
        why = "unsupported RGB-to-raw method";
        status.category = FJ_STATUS_UNSUPPORTED_INPUT;
        return false;
    }
    p.method = (int)ex.method;
    p.input_color_space = (int)ex.input_color_space;
    p.decode_cctf = (ex.flags & FJ_FILM_DECODE_CCTF) ? 1 : 0;
    p.adapt_input = (ex.flags & FJ_FILM_ADAPT_INPUT) ? 1 : 0;
    std::memcpy(p.input_rgb_to_xyz, ex.input_rgb_to_xyz, sizeof(p.input_rgb_to_xyz));
    std::memcpy(p.input_xyz_adapt, ex.input_xyz_adapt, sizeof(p.input_xyz_adapt));
    std::memcpy(p.xyz_to_linear_srgb, ex.xyz_to_linear_srgb, sizeof(p.xyz_to_linear_srgb));
    p.mallett_midgray_scale = ex.mallett_green_midgray_scale;
    const float manual = std::exp2(ex.manual_exposure_ev);
    if (!std::isfinite(ex.manual_exposure_ev) || !std::isfinite(manual) || !(manual > 0.0f) ||
        !std::isfinite(ex.route_correction_scale) || !(ex.route_correction_scale > 0.0f)) {
        why = "film exposure scale is not a positive finite number";
        return false;
    }
    p.manual_exposure_scale = manual;
    p.route_correction_scale = ex.route_correction_scale;
    if (!span_ok(ex.sensitivity_rgb, (size_t)kSpectralSamples * 3)) {
        why = "film_exposure.sensitivity_rgb must hold 81*3 floats";
        return false;
    }
    cudaError_t e = cudaSuccess;
    if (ex.method == FJ_RAW_MALLETT_2019) {
        if (!span_ok(ex.mallett_illuminant, kSpectralSamples) || !span_ok(ex.mallett_basis, kSpectralSamples * 3)) {
            why = "Mallett reconstruction needs an 81-sample illuminant and 81x3 basis";
            return false;
        }
        std::vector<float> sens((size_t)3 * kSpectralSamples);
        for (int i = 0; i < kSpectralSamples; ++i) {
            sens[i] = ex.sensitivity_rgb.data[i * 3 + 2];
            sens[kSpectralSamples + i] = ex.sensitivity_rgb.data[i * 3 + 1];
            sens[2 * kSpectralSamples + i] = ex.sensitivity_rgb.data[i * 3 + 0];
        }
        if ((e = upload(&r.film_sens_bgr, sens.data(), sens.size() * 4, stream)) != cudaSuccess ||
            (e = upload(&r.mallett_basis, ex.mallett_basis.data, kSpectralSamples * 3 * 4, stream)) != cudaSuccess ||
            (e = upload(&r.mallett_illum, ex.mallett_illuminant.data, kSpectralSamples * 4, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            goto cuda_fail;
        }
    } else {
        if (!span_ok(ex.tc_lut_rgba, (size_t)kTcLutExtent * kTcLutExtent * 4)) {
            why = "film_exposure.tc_lut_rgba must hold 192*192*4 floats";
            return false;
        }
        if ((e = upload(&r.tc_lut, ex.tc_lut_rgba.data, ex.tc_lut_rgba.count * 4, stream)) != cudaSuccess) goto cuda_fail;
    }
    p.tc_lut = reinterpret_cast<const float4*>(r.tc_lut);
    p.mallett_basis = r.mallett_basis;
    p.mallett_illum = r.mallett_illum;
    p.film_sens_bgr = r.film_sens_bgr;

    {
        // ---- development curves ----
        const FjFilmDevelopment& dv = h.film_development;
        const size_t n = dv.log_exposure.count;
        if (n < 2 || n > (size_t)kMaxCurveSamples || !span_ok(dv.density_rgb, n * 3)) {
            why = "film_development curves must hold N>=2 samples with N*3 densities";
            return false;
        }
        std::vector<float>& blob = r.blob;
        blob.clear();
        const int xoff = (int)blob.size();
        blob.insert(blob.end(), dv.log_exposure.data, dv.log_exposure.data + n);
        int yoff[3];
        for (int bgr = 0; bgr < 3; ++bgr) {
            yoff[bgr] = (int)blob.size();
            const int rgb = 2 - bgr;
            for (size_t i = 0; i < n; ++i) blob.push_back(dv.density_rgb.data[i * 3 + rgb]);
            p.film_curve[bgr] = CurveRef{xoff, yoff[bgr], (int)n};
            p.gamma_bgr[bgr] = dv.gamma_rgb[rgb];
        }
        // Sublayer density curves [layer][CMY] for the grain's layer model, kept
        // when all nine are present with the development's sample count.
        bool layers = true;
        for (int l = 0; l < 3; ++l)
            for (int c = 0; c < 3; ++c) layers = layers && dv.density_layers[l][c].data && dv.density_layers[l][c].count == n;
        if (layers) {
            std::vector<float> lc(9 * n);
            for (int l = 0; l < 3; ++l)
                for (int c = 0; c < 3; ++c)
                    std::copy(dv.density_layers[l][c].data, dv.density_layers[l][c].data + n, lc.begin() + (l * 3 + c) * n);
            if ((e = upload(&r.layer_curves, lc.data(), lc.size() * 4, stream)) != cudaSuccess ||
                (e = cudaStreamSynchronize(stream)) != cudaSuccess)
                goto cuda_fail;
            r.layer_n = (int)n;
        }
        const FjDirCouplers& dir = h.dir_couplers;
        if (dir.mode > FJ_DIR_POSITIVE_RECEIVER_LANGMUIR) {
            why = "unsupported DIR mode";
            status.category = FJ_STATUS_UNSUPPORTED_INPUT;
            return false;
        }
        p.dir_mode = (int)dir.mode;
        if (dir.mode != FJ_DIR_INACTIVE) {
            for (int bgr = 0; bgr < 3; ++bgr) {
                const int rgb = 2 - bgr;
                if (!span_ok(dir.compensated_axes_rgb[rgb], n)) {
                    why = "dir_couplers.compensated_axes_rgb must match the density sample count";
                    return false;
                }
                const int ax = (int)blob.size();
                blob.insert(blob.end(), dir.compensated_axes_rgb[rgb].data, dir.compensated_axes_rgb[rgb].data + n);
                p.dir_curve[bgr] = CurveRef{ax, yoff[bgr], (int)n};
                for (int rb = 0; rb < 3; ++rb) p.dir_m[bgr * 3 + rb] = dir.matrix_rgb[(2 - bgr) * 3 + (2 - rb)];
                p.dir_dmax[bgr] = dir.density_max_rgb[rgb];
                p.dir_dref[bgr] = dir.density_ref_rgb[rgb];
                p.dir_donor_k[bgr] = dir.donor_k_rgb[rgb];
                p.dir_receiver_cref[bgr] = dir.receiver_c_ref_rgb[rgb];
                p.dir_receiver_kr[bgr] = dir.receiver_kr_rgb[rgb];
            }
        }

        // ---- print ----
        if (print) {
            const FjPrint& pr = h.print;
            const size_t np = pr.log_exposure.count;
            if (np < 2 || np > (size_t)kMaxCurveSamples || !span_ok(pr.density_cmy, np * 3) ||
                !span_ok(pr.film_density_cmy, kSpectralSamples * 3) || !span_ok(pr.film_base_density, kSpectralSamples) ||
                !span_ok(pr.sensitivity_cmy, kSpectralSamples * 3) || !span_ok(pr.main_illuminant, kSpectralSamples)) {
                why = "print tables are incomplete";
                return false;
            }
            if (!std::isfinite(pr.exposure) || pr.exposure < 0.0f || !std::isfinite(pr.normalizer) ||
                !(pr.normalizer > 0.0f)) {
                why = "print exposure/normalizer must be finite and positive";
                return false;
            }
            const int px = (int)blob.size();
            blob.insert(blob.end(), pr.log_exposure.data, pr.log_exposure.data + np);
            for (int c = 0; c < 3; ++c) {
                const int off = (int)blob.size();
                for (size_t i = 0; i < np; ++i) blob.push_back(pr.density_cmy.data[i * 3 + c]);
                p.print_curve[c] = CurveRef{px, off, (int)np};
            }
            p.print_exposure = pr.exposure;
            const float pcorr = h.scanner_correction.exposure_scale;
            if (!std::isfinite(pcorr) || !(pcorr > 0.0f)) {
                why = "scanner_correction.exposure_scale must be finite and positive on print routes";
                return false;
            }
            p.print_route_correction = pcorr;
            p.print_midgray = pr.normalizer;
            const bool preflash = (pr.flags & FJ_PRINT_PREFLASH) != 0;
            p.print_preflash_exposure = preflash ? pr.preflash_exposure : 0.0f;
            for (int c = 0; c < 3; ++c) p.print_preflash_raw[c] = preflash ? pr.preflash_raw_cmy[c] : 0.0f;
            const float kLog2Of10 = 3.32192809488736234787f;
            int count = 0;
            for (int l = 0; l < kSpectralSamples; ++l) {
                const float s[3] = {pr.sensitivity_cmy.data[l * 3], pr.sensitivity_cmy.data[l * 3 + 1],
                                    pr.sensitivity_cmy.data[l * 3 + 2]};
                if (std::isnan(s[0]) && std::isnan(s[1]) && std::isnan(s[2])) continue;
                const float il = pr.main_illuminant.data[l];
                // a NaN dye or base density (or illuminant) makes the transmittance NaN
                // for every pixel, and the print integral drops NaN transmittances
                // (src/Cuda/JuicerCudaDeviceHelpers.cuh:860-864): the wavelength is idle
                const float* eps = pr.film_density_cmy.data + l * 3;
                if (std::isnan(eps[0]) || std::isnan(eps[1]) || std::isnan(eps[2]) ||
                    std::isnan(pr.film_base_density.data[l]) || std::isnan(il))
                    continue;
                for (int c = 0; c < 3; ++c) p.spectral.nd[count][c] = -(pr.film_density_cmy.data[l * 3 + c] * kLog2Of10);
                // the film base transmits the same 2^nd3 at every pixel: it is folded into
                // the wavelength's weights, so the per-pixel exponent is d . nd alone
                const float nd3 = -(pr.film_base_density.data[l] * kLog2Of10);
                const double base_t = std::exp2((double)nd3);
                p.spectral.nd[count][3] = 0.0f;
                for (int c = 0; c < 3; ++c)
                    p.spectral.sens[count][c] =
                        (std::isnan(s[c]) || std::isnan(il)) ? 0.0f : (float)((double)s[c] * (double)il * base_t);
                ++count;
            }
            p.spectral.count = count;
            for (int l = count; l < kSpectralSamples; ++l) {
                p.spectral.nd[l][0] = p.spectral.nd[l][1] = p.spectral.nd[l][2] = 0.0f;
                p.spectral.nd[l][3] = -INFINITY;
                p.spectral.sens[l][0] = p.spectral.sens[l][1] = p.spectral.sens[l][2] = 0.0f;
            }
        }
        for (CurveRef* c : {&p.film_curve[0], &p.film_curve[1], &p.film_curve[2], &p.dir_curve[0], &p.dir_curve[1],
                            &p.dir_curve[2], &p.print_curve[0], &p.print_curve[1], &p.print_curve[2]})
            set_curve_guess(blob, *c);
        while (blob.size() % 4) blob.push_back(0.0f);
        if ((e = upload(&r.curves, blob.data(), blob.size() * 4, stream)) != cudaSuccess) goto cuda_fail;
        p.curve_blob = r.curves;
        p.curve_blob_floats = (int)blob.size();
    }

    {
        // ---- scanner ----
        const FjDensityBounds& b = h.scanner_bounds;
        p.scan_medium_negative = print ? 0 : 1;
        for (int c = 0; c < 3; ++c) {
            p.scan_min_cmy[c] = print ? b.min_cmy[c] : -b.min_cmy[c];
            p.scan_inv_span_cmy[c] = b.inv_span_cmy[c];
        }
        const FjScannerSpectra& sp = h.scanner_spectra;
        const int res = (int)h.scanner_lut.resolution;
        if (res < 2 || res > 64 || !span_ok(sp.dye_c, kSpectralSamples) || !span_ok(sp.dye_m, kSpectralSamples) ||
            !span_ok(sp.dye_y, kSpectralSamples) || !span_ok(sp.weighted_x, kSpectralSamples) ||
            !span_ok(sp.weighted_y, kSpectralSamples) || !span_ok(sp.weighted_z, kSpectralSamples) ||
            (sp.base_density.count != 0 && !span_ok(sp.base_density, kSpectralSamples))) {
            why = "scanner spectra or LUT resolution are malformed";
            return false;
        }
        LutSource ls{};
        ls.eps_c = sp.dye_c.data;
        ls.eps_m = sp.dye_m.data;
        ls.eps_y = sp.dye_y.data;
        ls.wx = sp.weighted_x.data;
        ls.wy = sp.weighted_y.data;
        ls.wz = sp.weighted_z.data;
        ls.baseline = sp.base_density.count ? sp.base_density.data : nullptr;
        ls.k = kSpectralSamples;
        ls.inv_yn = sp.inverse_y_normalization;
        for (int c = 0; c < 3; ++c) {
            ls.range_min_cmy[c] = p.scan_min_cmy[c];
            ls.inverse_span_cmy[c] = p.scan_inv_span_cmy[c];
        }
        ls.medium = print ? 1 : 0;
        ls.resolution = res;
        if ((e = build_scanner_lut(ls, r.lut, &r.lut_spectra, stream)) != cudaSuccess) goto cuda_fail;
        unsigned fail = 0;
        if ((e = cudaMemcpy(&fail, r.lut.failure, sizeof(unsigned), cudaMemcpyDeviceToHost)) != cudaSuccess)
            goto cuda_fail;
        if (fail) {
            why = "scanner LUT build produced a non-finite log2 XYZ";
            return false;
        }
        p.scan_res = res;
        p.scan_nodes = r.lut.packed_nodes;
        p.scan_cells = r.lut.packed_cells;
        const FjScannerCorrection& cr = h.scanner_correction;
        p.correction_active = (cr.flags & FJ_CORRECTION_ACTIVE) ? 1 : 0;
        p.correction_slope = cr.xyz_slope;
        p.correction_offset = cr.xyz_offset;
    }

    {
        // ---- output colour ----
        const FjOutputColor& oc = h.output_color;
        const uint32_t known = FJ_COLOR_ENCODE_CCTF | FJ_COLOR_INPUT_IS_OUTPUT_SPACE | FJ_COLOR_GAMUT_COMPRESSION;
        if (oc.color_space > FJ_OUTPUT_REC709 || (oc.flags & ~known) != 0 ||
            oc.encoding.schema != FJ_OUTPUT_ENCODING_SCHEMA || oc.encoding.cctf_kind > FJ_CCTF_DWG_INTERMEDIATE) {
            why = "output colour record is malformed";
            return false;
        }
        std::memcpy(p.cat02, oc.cat02, sizeof(p.cat02));
        std::memcpy(p.scan_illuminant_xyz, oc.illuminant_xyz, sizeof(p.scan_illuminant_xyz));
        std::memcpy(p.xyz_to_rgb, oc.xyz_to_rgb, sizeof(p.xyz_to_rgb));
        p.gamut_active = (oc.flags & FJ_COLOR_GAMUT_COMPRESSION) ? 1 : 0;
        if (p.gamut_active) {
            if (!span_ok(oc.gamut_cmax, (size_t)kGamutLightness * kGamutHue)) {
                why = "output gamut compression needs the 64x720 boundary table";
                return false;
            }
            if ((e = upload(&r.gamut_cmax, oc.gamut_cmax.data, oc.gamut_cmax.count * 4, stream)) != cudaSuccess)
                goto cuda_fail;
        }
        p.gamut_cmax = r.gamut_cmax;
        std::memcpy(p.gamut_native_to_xyz, oc.native_rgb_to_d65_xyz, sizeof(p.gamut_native_to_xyz));
        std::memcpy(p.gamut_xyz_to_native, oc.d65_xyz_to_native_rgb, sizeof(p.gamut_xyz_to_native));
        std::memcpy(p.gamut_lightness_knee, oc.lightness_knee, sizeof(p.gamut_lightness_knee));
        std::memcpy(p.gamut_chroma_knee, oc.chroma_knee, sizeof(p.gamut_chroma_knee));
        p.encode_input_is_output = (oc.flags & FJ_COLOR_INPUT_IS_OUTPUT_SPACE) ? 1 : 0;
        p.encode_apply_cctf = (oc.flags & FJ_COLOR_ENCODE_CCTF) ? 1 : 0;
        std::memcpy(p.encode_dwg_to_output, oc.encoding.dwg_to_output, sizeof(p.encode_dwg_to_output));
        p.cctf_kind = (int)oc.encoding.cctf_kind;
        p.cctf_gamma = oc.encoding.gamma;
        p.cctf_a = oc.encoding.a;
        p.cctf_b = oc.encoding.b;
        p.cctf_c = oc.encoding.c;
        p.cctf_d = oc.encoding.d;
        p.cctf_linear_cutoff = oc.encoding.linear_cutoff;
    }

    if ((e = cudaMalloc(&r.meter_scratch, meter_scratch_bytes())) != cudaSuccess) goto cuda_fail;
    if ((e = cudaMemsetAsync(r.meter_scratch, 0, meter_scratch_bytes(), stream)) != cudaSuccess) goto cuda_fail;
    if ((e = cudaMalloc(&r.flags, sizeof(unsigned))) != cudaSuccess) goto cuda_fail;
    if ((e = cudaMemsetAsync(r.flags, 0, sizeof(unsigned), stream)) != cudaSuccess) goto cuda_fail;
    p.error_flags = r.flags;
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) goto cuda_fail;
    status = FjStatus{FJ_STATUS_SUCCESS, FJ_API_NONE, 0};
    return true;

cuda_fail:
    why = std::string("CUDA failure while preparing recipe tables: ") + cudaGetErrorString(e);
    status = FjStatus{e == cudaErrorMemoryAllocation ? FJ_STATUS_ALLOCATION_FAILURE : FJ_STATUS_CUDA_FAILURE,
                      FJ_API_CUDA_RUNTIME, (int32_t)e};
    r.release();
    return false;
}

} // namespace fjb
