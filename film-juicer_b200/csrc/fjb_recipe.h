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
    ScannerLutDevice lut{};
    void release() noexcept;
};

bool create_recipe(const FjPreparedHostData& h, cudaStream_t stream, Recipe& r, std::string& why, FjStatus& status);

cudaError_t alloc_scanner_lut(int r, ScannerLutDevice& lut);
void free_scanner_lut(ScannerLutDevice& lut);
cudaError_t build_scanner_lut(const LutSource& src, ScannerLutDevice& lut, double** doubles, cudaStream_t stream);

} // namespace fjb
