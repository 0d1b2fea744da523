// fjb_api.cpp -- extern "C" boundary of libjuicer_b200.so.
//
// fj_cuda_* restate the lifecycle and render contract of the reference's native
// adapter (native/juicer_cuda_api.cpp:245-600): one owner handle, typed FjStatus
// results, diagnostics written into the caller's FjErrorBuffer (always NUL
// terminated, truncation never changes the status), no exception crossing the
// boundary, abort queried at bounded checkpoints, synchronisation of the frame
// stream when the host did not supply one (native/juicer_cuda_api.cpp:475-479).
// The stage schedule of fj_cuda_render lives in fjb_schedule.cpp.
#include <cuda_runtime.h>

#include <atomic>

#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "../../include/juicer_cuda_api.h"
#include "fjb_internal.h"
#include "fjb_recipe.h"
#include "fjb_optics.h"
#include "fjb_launches.h"
#include "fjb_schedule.h"

namespace fjb {

namespace {
std::atomic<unsigned long long> g_launches{0};
}

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void write_error(FjErrorBuffer* error, const std::string& text) {
    if (!error) return;
    error->length = 0;
    if (!error->data || error->capacity == 0) return;
    const size_t n = text.size() < error->capacity - 1 ? text.size() : error->capacity - 1;
    std::memcpy(error->data, text.data(), n);
    error->data[n] = '\0';
    error->length = n;
}

FjStatus ok_status() { return FjStatus{FJ_STATUS_SUCCESS, FJ_API_NONE, 0}; }

FjStatus fail_status(uint32_t category, FjErrorBuffer* error, const std::string& text) {
    write_error(error, text);
    return FjStatus{category, FJ_API_NONE, 0};
}

FjStatus cuda_status(cudaError_t e, FjErrorBuffer* error, const char* where) {
    write_error(error, std::string(where) + ": " + cudaGetErrorString(e));
    uint32_t cat = FJ_STATUS_CUDA_FAILURE;
    if (e == cudaErrorMemoryAllocation) cat = FJ_STATUS_ALLOCATION_FAILURE;
    return FjStatus{cat, FJ_API_CUDA_RUNTIME, (int32_t)e};
}

} // namespace fjb

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

namespace {

bool valid_components(uint32_t c) { return c == 3 || c == 4; }

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

} // namespace

extern "C" {

uint64_t fjb_kernel_launches(void) { return (uint64_t)fjb::g_launches.load(std::memory_order_relaxed); }

FjStatus fjb_recipe_create(const FjPreparedHostData* prepared, void* stream, FjbRecipe** out_recipe,
                           FjErrorBuffer* error) {
    try {
        if (!prepared || !out_recipe) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        *out_recipe = nullptr;
        auto* holder = new (std::nothrow) FjbRecipe();
        if (!holder) return fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "host allocation failed");
        cudaGetDevice(&holder->device);
        std::string why;
        FjStatus st{};
        if (!fjb::create_recipe(*prepared, as_stream(stream), holder->r, why, st)) {
            holder->r.release();
            delete holder;
            write_error(error, why);
            return st;
        }
        *out_recipe = holder;
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_recipe_create");
    }
}

FjStatus fjb_recipe_destroy(FjbRecipe* recipe, FjErrorBuffer* error) {
    if (!recipe) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null recipe");
    recipe->r.release();
    delete recipe;
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_recipe_set_exposure_scale_device(FjbRecipe* recipe, const float* device_scale, FjErrorBuffer* error) {
    if (!recipe) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null recipe");
    recipe->r.params.auto_exposure_scale = device_scale;
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_recipe_set_print_form(FjbRecipe* recipe, int32_t form, FjErrorBuffer* error) {
    if (!recipe) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null recipe");
    if (form != FJB_PRINT_FP32 && form != FJB_PRINT_TENSOR && form != FJB_PRINT_TENSOR_SPLIT)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unknown print form");
    recipe->r.params.print_form = form;
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_recipe_clear_flags(FjbRecipe* recipe, void* stream, FjErrorBuffer* error) {
    if (!recipe) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null recipe");
    cudaError_t e = cudaMemsetAsync(recipe->r.flags, 0, sizeof(unsigned), as_stream(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "clear flags");
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_recipe_read_flags(FjbRecipe* recipe, void* stream, uint32_t* out_flags, FjErrorBuffer* error) {
    if (!recipe || !out_flags) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    unsigned v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, recipe->r.flags, sizeof(unsigned), cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "read flags");
    *out_flags = v;
    write_error(error, "");
    return ok_status();
}

static FjStatus launch_stage(FjbRecipe* recipe, fjb::PixelParams& p, fjb::PixelStage stage, void* stream,
                             FjErrorBuffer* error) {
    if (p.route == fjb::kRoutePrint && p.print_form != fjb::kPrintFp32 && !p.print_done &&
        (stage == fjb::PixelStage::DensityToOutput || stage == fjb::PixelStage::DensityToLinearRgb)) {
        // the tensor-core form hands the spectral integral to the FP32 epilogue in planes
        cudaError_t e = recipe->r.ensure_tc_raw((size_t)p.width * (size_t)p.height);
        if (e != cudaSuccess) return cuda_status(e, error, "tensor-core print planes");
        p.tc_raw = recipe->r.tc_raw;
    }
    cudaError_t e = fjb::launch_pixel_chain(p, stage, as_stream(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "pixel chain launch");
    (void)recipe;
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_render_pixels(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, float* dst,
                           ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                           void* stream, FjErrorBuffer* error) {
    if (!recipe || !src || !dst) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (!valid_components(components) || width < 0 || height < 0 || src_row_bytes <= 0 || dst_row_bytes <= 0)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unsupported image geometry");
    fjb::PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src);
    p.dst = reinterpret_cast<char*>(dst);
    p.src_row_bytes = src_row_bytes;
    p.dst_row_bytes = dst_row_bytes;
    p.width = width;
    p.height = height;
    p.components = (int)components;
    return launch_stage(recipe, p, fjb::PixelStage::SourceToOutput, stream, error);
}

FjStatus fjb_camera_exposure(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, uint32_t components,
                             int32_t width, int32_t height, float* carrier_b, float* carrier_g, float* carrier_r,
                             ptrdiff_t carrier_stride, void* stream, FjErrorBuffer* error) {
    if (!recipe || !src || !carrier_b || !carrier_g || !carrier_r)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (!valid_components(components) || width < 0 || height < 0 || carrier_stride < width)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unsupported image geometry");
    fjb::PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src);
    p.src_row_bytes = src_row_bytes;
    p.width = width;
    p.height = height;
    p.components = (int)components;
    cudaError_t e = fjb::launch_camera_exposure(p, carrier_b, carrier_g, carrier_r, carrier_stride, as_stream(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "camera exposure launch");
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_capture_density(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, uint32_t components,
                             const float* carrier_b, const float* carrier_g, const float* carrier_r,
                             ptrdiff_t carrier_stride, int32_t width, int32_t height, float* density_c,
                             float* density_m, float* density_y, void* stream, FjErrorBuffer* error) {
    if (!recipe || !density_c || !density_m || !density_y)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    const bool carrier = carrier_b && carrier_g && carrier_r;
    if (!carrier && (!src || !valid_components(components)))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "capture density needs a source image or carrier planes");
    fjb::PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src);
    p.src_row_bytes = src_row_bytes;
    p.components = (int)components;
    p.width = width;
    p.height = height;
    p.carrier_b = carrier_b;
    p.carrier_g = carrier_g;
    p.carrier_r = carrier_r;
    p.carrier_stride = carrier_stride;
    p.density_c = density_c;
    p.density_m = density_m;
    p.density_y = density_y;
    return launch_stage(recipe, p, carrier ? fjb::PixelStage::CarrierToDensity : fjb::PixelStage::SourceToDensity,
                        stream, error);
}

FjStatus fjb_render_carrier(FjbRecipe* recipe, const float* carrier_b, const float* carrier_g,
                            const float* carrier_r, ptrdiff_t carrier_stride, const float* src_alpha_source,
                            ptrdiff_t src_row_bytes, float* dst, ptrdiff_t dst_row_bytes, int32_t width,
                            int32_t height, uint32_t components, void* stream, FjErrorBuffer* error) {
    if (!recipe || !carrier_b || !carrier_g || !carrier_r || !dst)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (!valid_components(components)) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "components");
    fjb::PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src_alpha_source);
    p.src_row_bytes = src_row_bytes;
    p.dst = reinterpret_cast<char*>(dst);
    p.dst_row_bytes = dst_row_bytes;
    p.width = width;
    p.height = height;
    p.components = (int)components;
    p.carrier_b = carrier_b;
    p.carrier_g = carrier_g;
    p.carrier_r = carrier_r;
    p.carrier_stride = carrier_stride;
    return launch_stage(recipe, p, fjb::PixelStage::CarrierToOutput, stream, error);
}

FjStatus fjb_render_from_density(FjbRecipe* recipe, const float* density_c, const float* density_m,
                                 const float* density_y, const float* src, ptrdiff_t src_row_bytes, float* dst,
                                 ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                 void* stream, FjErrorBuffer* error) {
    if (!recipe || !density_c || !density_m || !density_y || !dst)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (!valid_components(components)) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "components");
    fjb::PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src);
    p.src_row_bytes = src_row_bytes;
    p.dst = reinterpret_cast<char*>(dst);
    p.dst_row_bytes = dst_row_bytes;
    p.width = width;
    p.height = height;
    p.components = (int)components;
    p.scan_density_c = density_c;
    p.scan_density_m = density_m;
    p.scan_density_y = density_y;
    return launch_stage(recipe, p, fjb::PixelStage::DensityToOutput, stream, error);
}

FjStatus fjb_print_raw(FjbRecipe* recipe, const float* density_c, const float* density_m, const float* density_y,
                       float* raw_c, float* raw_m, float* raw_y, int32_t width, int32_t height, void* stream,
                       FjErrorBuffer* error) {
    if (!recipe || !density_c || !density_m || !density_y || !raw_c || !raw_m || !raw_y)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (recipe->r.params.route != fjb::kRoutePrint)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "the recipe has no print stage");
    if (width < 0 || height < 0) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unsupported image geometry");
    fjb::PixelParams p = recipe->r.params;
    p.width = width;
    p.height = height;
    p.scan_density_c = density_c;
    p.scan_density_m = density_m;
    p.scan_density_y = density_y;
    p.lin_r = raw_c;
    p.lin_g = raw_m;
    p.lin_b = raw_y;
    p.film_dust = nullptr;
    return launch_stage(recipe, p, fjb::PixelStage::DensityToPrintRaw, stream, error);
}

FjStatus fjb_enlarger_linear_exposure(FjbRecipe* recipe, const float* density_c, const float* density_m,
                                      const float* density_y, const float* dust, float* linear_c, float* linear_m,
                                      float* linear_y, int32_t width, int32_t height, void* stream,
                                      FjErrorBuffer* error) {
    if (!recipe || !density_c || !density_m || !density_y || !linear_c || !linear_m || !linear_y)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (recipe->r.params.route != fjb::kRoutePrint)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "the recipe has no print stage");
    if (width < 0 || height < 0) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unsupported image geometry");
    fjb::PixelParams p = recipe->r.params;
    p.width = width;
    p.height = height;
    p.scan_density_c = density_c;
    p.scan_density_m = density_m;
    p.scan_density_y = density_y;
    p.film_dust = dust;
    p.lin_r = linear_c;
    p.lin_g = linear_m;
    p.lin_b = linear_y;
    return launch_stage(recipe, p, fjb::PixelStage::DensityToEnlargerLinear, stream, error);
}

FjStatus fjb_enlarger_develop(FjbRecipe* recipe, const float* linear_c, const float* linear_m, const float* linear_y,
                              float* density_c, float* density_m, float* density_y, int32_t width, int32_t height,
                              void* stream, FjErrorBuffer* error) {
    if (!recipe || !density_c || !density_m || !density_y || !linear_c || !linear_m || !linear_y)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (recipe->r.params.route != fjb::kRoutePrint)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "the recipe has no print stage");
    if (width < 0 || height < 0) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unsupported image geometry");
    fjb::PixelParams p = recipe->r.params;
    p.width = width;
    p.height = height;
    p.scan_density_c = linear_c;
    p.scan_density_m = linear_m;
    p.scan_density_y = linear_y;
    p.density_c = density_c;
    p.density_m = density_m;
    p.density_y = density_y;
    return launch_stage(recipe, p, fjb::PixelStage::EnlargerLinearToPrintDensity, stream, error);
}

FjStatus fjb_render_from_print_density(FjbRecipe* recipe, const float* density_c, const float* density_m,
                                       const float* density_y, const float* src, ptrdiff_t src_row_bytes, float* dst,
                                       ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                       void* stream, FjErrorBuffer* error) {
    if (!recipe || !density_c || !density_m || !density_y || !dst)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (!valid_components(components)) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "components");
    if (recipe->r.params.route != fjb::kRoutePrint)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "the recipe has no print stage");
    fjb::PixelParams p = recipe->r.params;
    p.print_done = 1;
    p.film_dust = nullptr;
    p.src = reinterpret_cast<const char*>(src);
    p.src_row_bytes = src_row_bytes;
    p.dst = reinterpret_cast<char*>(dst);
    p.dst_row_bytes = dst_row_bytes;
    p.width = width;
    p.height = height;
    p.components = (int)components;
    p.scan_density_c = density_c;
    p.scan_density_m = density_m;
    p.scan_density_y = density_y;
    return launch_stage(recipe, p, fjb::PixelStage::DensityToOutput, stream, error);
}

FjStatus fjb_auto_exposure(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, uint32_t components,
                           const FjAutoExposure* meter, float* device_scale, void* stream, FjErrorBuffer* error) {
    if (!recipe || !src || !meter || !device_scale) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    fjb::MeterSpec m{};
    std::string why;
    if (!valid_components(components) || !fjb::meter_spec_from(*meter, m, why))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, why.empty() ? "components" : why);
    fjb::PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src);
    p.src_row_bytes = src_row_bytes;
    p.components = (int)components;
    cudaError_t e = fjb::launch_auto_exposure(p, m, recipe->r.meter_scratch, device_scale, as_stream(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "auto exposure launch");
    write_error(error, "");
    return ok_status();
}

size_t fjb_scatter_halation_scratch_bytes(int32_t width, int32_t height) {
    if (width <= 0 || height <= 0) return 0;
    return fjb::halation_scratch_floats(width, height) * sizeof(float);
}

FjStatus fjb_scatter_halation(const FjScatterHalation* halation, float* carrier_r, float* carrier_g,
                              float* carrier_b, ptrdiff_t stride, int32_t width, int32_t height, float* scratch,
                              size_t scratch_bytes, void* stream, FjErrorBuffer* error) {
    try {
        if (!halation || !carrier_r || !carrier_g || !carrier_b)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (width <= 0 || height <= 0) {
            write_error(error, "");
            return ok_status();
        }
        if (stride < width) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "carrier stride below width");
        if (!scratch || scratch_bytes < fjb_scatter_halation_scratch_bytes(width, height))
            return fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "scatter/halation scratch is too small");
        float* planes[3] = {carrier_r, carrier_g, carrier_b};
        std::string why;
        cudaError_t e = cudaSuccess;
        if (!fjb::scatter_halation(*halation, planes, stride, width, height, scratch, as_stream(stream), why, e)) {
            if (e != cudaSuccess) return cuda_status(e, error, why.c_str());
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        }
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_scatter_halation");
    }
}

FjStatus fjb_scanner_lut_build_host(const FjbScannerLutInput* in, float* log2_xyz, float* slope_c, float* slope_m,
                                    float* slope_y, float* cell_min, float* cell_max, FjErrorBuffer* error) {
    try {
        if (!in || !log2_xyz || !slope_c || !slope_m || !slope_y || !cell_min || !cell_max)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        const int r = (int)in->resolution;
        const int k = in->sample_count;
        if (r < 2 || r > 64) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "resolution must be 2..64");
        if (k <= 0 || in->eps_c.count != (size_t)k || in->eps_m.count != (size_t)k || in->eps_y.count != (size_t)k ||
            in->weighted_x.count != (size_t)k || in->weighted_y.count != (size_t)k ||
            in->weighted_z.count != (size_t)k || (in->has_baseline && in->baseline_min.count != (size_t)k))
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "spectral spans must all hold sample_count floats");
        fjb::LutSource src{};
        src.eps_c = in->eps_c.data;
        src.eps_m = in->eps_m.data;
        src.eps_y = in->eps_y.data;
        src.wx = in->weighted_x.data;
        src.wy = in->weighted_y.data;
        src.wz = in->weighted_z.data;
        src.baseline = in->has_baseline ? in->baseline_min.data : nullptr;
        src.k = k;
        src.inv_yn = in->inv_yn;
        for (int c = 0; c < 3; ++c) {
            src.range_min_cmy[c] = in->range_min_cmy[c];
            src.inverse_span_cmy[c] = in->inverse_span_cmy[c];
        }
        src.medium = (int)in->medium;
        src.resolution = r;
        fjb::ScannerLutDevice lut{};
        double* spectra = nullptr;
        cudaStream_t s = nullptr;
        cudaError_t e = fjb::build_scanner_lut(src, lut, &spectra, s);
        const size_t nodes = (size_t)r * r * r * 3;
        const size_t cells = (size_t)(r - 1) * (r - 1) * (r - 1) * 3;
        unsigned failed = 0;
        if (e == cudaSuccess) e = cudaMemcpy(log2_xyz, lut.log2_xyz, nodes * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(slope_c, lut.slope_c, nodes * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(slope_m, lut.slope_m, nodes * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(slope_y, lut.slope_y, nodes * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(cell_min, lut.cell_min, cells * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(cell_max, lut.cell_max, cells * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(&failed, lut.failure, sizeof(unsigned), cudaMemcpyDeviceToHost);
        fjb::free_scanner_lut(lut);
        if (spectra) cudaFree(spectra);
        if (e != cudaSuccess) return cuda_status(e, error, "scanner LUT build");
        if (failed) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "scanner LUT produced non-finite log2 XYZ");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in scanner LUT build");
    }
}

} // extern "C"
