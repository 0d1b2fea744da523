// fjb_params.h -- device-side parameter blocks of the fused per-pixel render chain.
//
// One PixelParams block describes a prepared recipe for one frame. It travels to the
// kernel as a __grid_constant__ parameter (it lives in the constant bank, so the
// 81-wavelength print coefficients are read as FFMA constant operands with no load
// instruction). Curve samples are staged once per CTA into shared memory; the large
// tables (TC LUT, scanner PCHIP nodes, gamut boundary) stay in HBM/L2 and are read
// as 16-byte vectors.
#pragma once

#include <cstddef>
#include <cstdint>

namespace fjb {

constexpr int kSpectralSamples = 81;   // 380..780 nm in 5 nm steps
constexpr int kTcLutExtent = 192;      // TC LUT is 192 x 192 (x, y) nodes
constexpr int kGamutLightness = 64;    // output gamut boundary rows
constexpr int kGamutHue = 720;         // output gamut boundary columns
constexpr int kMaxCurveSamples = 1024; // upper bound for staged curves

enum Route : int { kRouteDirect = 0, kRoutePrint = 1 };
// The print exposure's 81-wavelength contraction: FP32 FMAs (the parity form) or BF16
// tensor-core tiles with FP32 accumulation (tcgen05), densities and coefficients as
// hi + lo BF16 pairs, transmittances as one BF16 (kPrintTensor) or a hi + lo pair
// (kPrintTensorSplit).
enum PrintForm : int { kPrintFp32 = 0, kPrintTensor = 1, kPrintTensorSplit = 2 };
constexpr unsigned kErrTensorWait = 1u << 16;
enum RawMethod : int { kHanatos = 0, kMallett = 1, kArctic = 2 };
enum DirModeDev : int { kDirInactive = 0, kDirNegativeDonor = 1, kDirPositiveReceiver = 2 };

// Offsets (in floats) of the curve samples inside the staged curve blob.
struct CurveRef {
    int x;   // offset of the ascending abscissa
    int y;   // offset of the ordinate
    int n;   // sample count (accepted domain is [0, n-1])
    int guess;    // 1: the abscissa is strictly increasing and close to uniform
    float x0;     // first abscissa
    float inv_dx; // (n - 1) / (x[n-1] - x[0])
};

// Print 81-lambda coefficients, pre-folded on the host:
//   nd[l]   = (-(eps_c, eps_m, eps_y) * log2(10), 0)     (so T = 2^(D . nd))
//   sens[l] = (sens_c, sens_m, sens_y) * filtered illuminant * 10^-base
// (the film base's transmittance is the same at every pixel, so it sits in the
// weights and the per-pixel exponent has the three dye terms only; nd[l][3] stays 0).
// Wavelengths whose three sensitivities are all NaN, or whose dye or base density or
// illuminant is NaN, are dropped and the remaining ones packed first; the unused tail
// slots hold (0, 0, 0, -inf) and zero sensitivities, so they contribute exactly +0 for
// finite densities. A NaN channel of a kept wavelength contributes zero.
struct PrintSpectral {
    float nd[kSpectralSamples][4];
    float sens[kSpectralSamples][3];
    int count;
};

struct PixelParams {
    // ---- frame ----
    const char* src;
    char* dst;
    long long src_row_bytes;
    long long dst_row_bytes;
    int width;
    int height;
    int components; // 3 or 4, same for source and destination
    int route;      // Route
    int print_form; // PrintForm: arithmetic of the 81-wavelength print contraction
    int print_done; // 1: the density planes already hold print density (enlarger diffusion), scan only

    // Optional carrier input: planar linear exposure (B, G, R) produced by the
    // camera optics stages. When set, exposure reconstruction is skipped.
    const float* carrier_b;
    const float* carrier_g;
    const float* carrier_r;
    long long carrier_stride; // floats per row

    // Optional materialised density output (capture stage only, C, M, Y planes).
    float* density_c;
    float* density_m;
    float* density_y;

    // ---- input colour + exposure reconstruction ----
    int input_color_space;
    int decode_cctf;
    int adapt_input;
    int method; // RawMethod
    float input_rgb_to_xyz[9];
    float input_xyz_adapt[9];
    float xyz_to_linear_srgb[9];
    float mallett_midgray_scale;
    const float4* tc_lut;        // [192][192] of (R, G, B, pad)
    const float* mallett_basis;  // [81][3]
    const float* mallett_illum;  // [81]
    const float* film_sens_bgr;  // [3][81] B, G, R relative sensitivity
    float manual_exposure_scale;
    float route_correction_scale;
    const float* auto_exposure_scale; // device scalar or null

    // ---- capture development ----
    float gamma_bgr[3];
    int dir_mode; // DirModeDev
    float dir_m[9]; // [donor BGR][receiver BGR]
    float dir_dmax[3];
    float dir_dref[3];
    float dir_donor_k[3];
    float dir_receiver_cref[3];
    float dir_receiver_kr[3];
    CurveRef film_curve[3]; // B, G, R: (log exposure, normalized density)
    CurveRef dir_curve[3];  // B, G, R: (compensated axis, normalized density)

    // Spatial DIR: filtered corrections (Y, M, C order of the B, G, R layers) and
    // cached raw log exposure (B, G, R). Used when dir_spatial != 0.
    int dir_spatial;
    const float* dir_filtered_y;
    const float* dir_filtered_m;
    const float* dir_filtered_c;
    const float* dir_log_raw_b;
    const float* dir_log_raw_g;
    const float* dir_log_raw_r;

    // Spatial-DIR source outputs: raw donor corrections (Y, M, C receivers) and raw
    // log exposure (B, G, R).
    float* dir_src_y;
    float* dir_src_m;
    float* dir_src_c;
    float* dir_src_log_b;
    float* dir_src_log_g;
    float* dir_src_log_r;

    // Optional density-plane input for the scan stage (after grain): C, M, Y planes.
    const float* scan_density_c;
    const float* scan_density_m;
    const float* scan_density_y;

    // ---- print ----
    float print_exposure;
    float print_route_correction;
    float print_preflash_exposure;
    float print_midgray;
    float print_preflash_raw[3];
    CurveRef print_curve[3]; // C, M, Y

    // ---- scanner ----
    int scan_medium_negative;
    float scan_min_cmy[3];
    float scan_inv_span_cmy[3];
    int scan_res;
    const float4* scan_nodes; // [(c*r+m)*r+y][3 outputs] of (value, slope_c, slope_m, slope_y)
    const float4* scan_cells; // [(c*s+m)*s+y][2] of (min xyz, max x), (max y, max z, 0, 0)
    int correction_active;
    float correction_slope;
    float correction_offset;
    // scanner post effects: glare percent plane added in XYZ (may be null), the scan
    // illuminant it is scaled by, and linear output-RGB planes written instead of the
    // encoded pixels when the stage stops before encoding
    const float* scan_glare;
    float scan_illuminant_xyz[3];
    float* lin_r;
    float* lin_g;
    float* lin_b;
    // film defects: dust transmittance plane (null when off), applied to the print
    // exposure on the print route and to the scanned XYZ on the direct route
    const float* film_dust;
    // print route, tensor-core form: the spectral integral (C, M, Y planes) computed by
    // the tensor-core kernel, read by the FP32 print / scan / output epilogue
    const float* print_raw_c;
    const float* print_raw_m;
    const float* print_raw_y;
    float* tc_raw; // scratch for those planes (3 x width x height floats), owned by the recipe
    // gate output (encoding of linear planes): weave resampling and the gate mask
    int weave_active;
    float weave_dx, weave_dy, weave_cos, weave_sin;
    const float* gate_mask; // gate_w x gate_h, sampled at (roi + pixel) / 2 - 1/4
    int gate_w, gate_h, roi_x, roi_y;

    // ---- output colour ----
    float cat02[9];
    float xyz_to_rgb[9];
    int gamut_active;
    const float* gamut_cmax; // [64][720]
    float gamut_native_to_xyz[9];
    float gamut_xyz_to_native[9];
    float gamut_lightness_knee[3];
    float gamut_chroma_knee[3];
    int encode_input_is_output;
    int encode_apply_cctf;
    float encode_dwg_to_output[9];
    int cctf_kind;
    float cctf_gamma, cctf_a, cctf_b, cctf_c, cctf_d, cctf_linear_cutoff;

    // ---- staged curves + error word ----
    const float* curve_blob;
    int curve_blob_floats;
    unsigned int* error_flags; // bit 0 scan failure, bit 8 DIR failure, bits 9..11 DIR channels,
                               // bit 16 a tensor-core wait gave up (print stage, tensor-core form)

    PrintSpectral spectral;
};

} // namespace fjb
