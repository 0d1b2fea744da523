// fjb_recipe.h -- device-resident tables of one prepared recipe.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/juicer_cuda_api.h"
#include "fjb_internal.h"

namespace fjb {

struct LutSource {
    const float* eps_c;
    const float* eps_m;
    const float* eps_y;
    const float* wx;
    const float* wy;
    const float* wz;
    const float* baseline; // may be null
    int k;
    float inv_yn;
    float range_min_cmy[3];
    float inverse_span_cmy[3];
    int medium;
    int resolution;
};

struct Recipe {
    PixelParams params{}; // device pointers filled, frame fields zero
    bool print = false;
    std::vector<float> blob;
    float* curves = nullptr;
    float* tc_lut = nullptr;
    float* mallett_basis = nullptr;
    float* mallett_illum = nullptr;
    float* film_sens_bgr = nullptr;
    float* gamut_cmax = nullptr;
    unsigned* flags = nullptr;
    double* lut_spectra = nullptr;
    void* meter_scratch = nullptr; // auto-exposure partial sums + ticket
    float* tc_raw = nullptr;       // tensor-core print form: spectral integral planes of the last frame
    size_t tc_raw_floats = 0;
    float* layer_curves = nullptr; // [layer][CMY] x layer_n sublayer density curves (grain), or null
    int layer_n = 0;
    bool positive_film = false;
    ScannerLutDevice lut{};
    void release() noexcept;
    // Grows tc_raw to 3 planes of `pixels` floats (stream-ordered reuse across frames).
    cudaError_t ensure_tc_raw(size_t pixels) noexcept;
};

bool create_recipe(const FjPreparedHostData& h, cudaStream_t stream, Recipe& r, std::string& why, FjStatus& status);

} // namespace fjb

// The C-ABI's opaque recipe handle.
struct FjbRecipe {
    fjb::Recipe r;
    int device = 0;
};

namespace fjb {

// FjAutoExposure -> metering grid; false (with a reason) for rejected records:
// median metering, empty preview or meter window, meter window outside the source.
inline bool meter_spec_from(const FjAutoExposure& a, MeterSpec& m, std::string& why) {
    if (a.method == FJ_METER_MEDIAN) {
        why = "median metering is not supported";
        return false;
    }
    if (a.method > FJ_METER_HIGHLIGHT_WEIGHTED) {
        why = "unknown metering method";
        return false;
    }
    if (a.preview_width <= 0 || a.preview_height <= 0 || a.meter_bounds.x2 <= a.meter_bounds.x1 ||
        a.meter_bounds.y2 <= a.meter_bounds.y1 || a.source_bounds.x2 <= a.source_bounds.x1 ||
        a.source_bounds.y2 <= a.source_bounds.y1) {
        why = "auto exposure preview or meter window is empty";
        return false;
    }
    m = MeterSpec{a.source_bounds.x1, a.source_bounds.y1, a.source_bounds.x2, a.source_bounds.y2,
                  a.meter_bounds.x1,  a.meter_bounds.y1,  a.meter_bounds.x2,  a.meter_bounds.y2,
                  a.preview_width,    a.preview_height,   (int)a.method};
    return true;
}

cudaError_t alloc_scanner_lut(int r, ScannerLutDevice& lut);
void free_scanner_lut(ScannerLutDevice& lut);
cudaError_t build_scanner_lut(const LutSource& src, ScannerLutDevice& lut, double** doubles, cudaStream_t stream);

} // namespace fjb
