// fjb_internal.h -- host-side declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "fjb_params.h"

namespace fjb {

constexpr int kPixelThreads = 256;
constexpr int kPixelBlocksPerSm = 4; // resident CTAs per SM when the occupancy query fails

enum class PixelStage : int {
    SourceToOutput = 0,   // monolithic frame: source RGB -> encoded output
    CarrierToOutput = 1,  // optics carrier planes -> encoded output
    SourceToDensity = 2,  // source RGB -> capture density planes
    CarrierToDensity = 3, // optics carrier planes -> capture density planes
    DensityToOutput = 4,  // (grained) capture density planes -> encoded output
    SourceToDirSource = 5,  // source RGB -> spatial-DIR raw corrections + log exposure
    CarrierToDirSource = 6, // carrier planes -> spatial-DIR raw corrections + log exposure
    DensityToLinearRgb = 7, // density planes -> linear output-RGB planes (+ glare), before encoding
    LinearRgbToOutput = 8,  // linear output-RGB planes -> encoded output
    DensityToPrintRaw = 9,  // density planes -> the print's spectral integral (C, M, Y) into lin_r/g/b
    RawToOutput = 10,       // print spectral integral planes (print_raw_*) -> encoded output
    RawToLinearRgb = 11,    // print spectral integral planes -> linear output-RGB planes
    DensityToEnlargerLinear = 12,      // capture density planes -> print-linear exposure (lin_r/g/b: C-, M-,
                                       // Y-forming), the enlarger diffusion's input
    EnlargerLinearToPrintDensity = 13, // diffused print-linear exposure (scan_density_*) -> print density
                                       // planes (density_*)
};

cudaError_t launch_pixel_chain(const PixelParams& p, PixelStage stage, cudaStream_t stream);

// The print stages from density planes (DensityToOutput, DensityToLinearRgb,
// DensityToPrintRaw) with the 81-wavelength contraction on the tensor cores
// (p.print_form kPrintTensor / kPrintTensorSplit, print route).
cudaError_t launch_print_tensor(const PixelParams& p, PixelStage stage, cudaStream_t stream);

// Camera linear exposure to planar B, G, R carrier planes (reference
// src/Cuda/Film/JuicerCudaFilmPipeline.cu:3103 camera_film_linear_exposure_kernel).
cudaError_t launch_camera_exposure(const PixelParams& p, float* b, float* g, float* r, long long stride,
                                   cudaStream_t stream);

// Scanner PCHIP LUT construction on the device in FP64 (reference
// rust/film-juicer-core/src/scanner/lut.rs:187-296).
struct ScannerLutSpec {
    const double* eps_c; // device, [k]
    const double* eps_m;
    const double* eps_y;
    const double* wx;
    const double* wy;
    const double* wz;
    const double* baseline; // device or null
    int k;
    double inv_yn;
    float range_min_cmy[3];
    float inverse_span_cmy[3];
    int medium; // 0 = negative, 1 = print/positive
    int resolution;
};

struct ScannerLutDevice {
    double* nodes;   // [r^3 * 3] log2 XYZ in FP64
    float* log2_xyz; // [r^3 * 3]
    float* slope_c;
    float* slope_m;
    float* slope_y;
    float* cell_min; // [(r-1)^3 * 3]
    float* cell_max;
    float4* packed_nodes; // [r^3 * 3]
    float4* packed_cells; // [(r-1)^3 * 2]
    unsigned int* failure; // non-finite node flag
};

cudaError_t launch_scanner_lut_build(const ScannerLutSpec& spec, const ScannerLutDevice& out, cudaStream_t stream);

// Auto-exposure metering (FJ_METER_* numbering).
enum MeterMethod : int {
    kMeterCenterWeighted = 0,
    kMeterAverage = 1,
    kMeterMedian = 2,
    kMeterPartial = 3,
    kMeterMatrix = 4,
    kMeterMultiZone = 5,
    kMeterHighlightWeighted = 6,
};
constexpr int kMeterBlocks = 148; // one CTA per SM at most

// Preview metering grid: `source` is the image's bounds, `meter` the metered window,
// preview_* the sample grid laid over the meter window (reference
// src/Cuda/JuicerCudaResources.h:169-184). p.src points at pixel (source_x1, source_y1).
struct MeterSpec {
    int source_x1, source_y1, source_x2, source_y2;
    int meter_x1, meter_y1, meter_x2, meter_y2;
    int preview_width, preview_height;
    int method;
};

size_t meter_scratch_bytes();
// Writes the exposure scale (float, device) for the frame. `scratch` holds
// meter_scratch_bytes() of device memory whose ticket word must be zero on entry (the
// kernel leaves it zero again).
cudaError_t launch_auto_exposure(const PixelParams& p, const MeterSpec& m, void* scratch, float* scale,
                                 cudaStream_t stream);

} // namespace fjb
