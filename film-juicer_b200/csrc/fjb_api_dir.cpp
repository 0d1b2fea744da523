// fjb_api_dir.cpp -- extern "C" entry points of the spatial-DIR stage.
//
// The stage order restates src/Cuda/Film/JuicerCudaFilmPipeline.cu:799-1060
// (build_spatial_dir_impl): raw donor corrections and raw log exposure per pixel,
// then the weighted Gaussian components on each correction plane; the filtered
// planes and the cached log exposure are then consumed by capture development
// (src/Cuda/JuicerCudaDeviceHelpers.cuh:1267-1328).
#include <cuda_runtime.h>

#include <string>

#include "../../include/juicer_b200.h"
#include "fjb_dir.h"
#include "fjb_internal.h"
#include "fjb_recipe.h"
#include "fjb_schedule.h"

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

namespace fjb {

cudaError_t dir_blur_planes(const DirPlan& plan, const float* const in[3], float* const out[3], int width, int height,
                            float* scratch, cudaStream_t s);

FjStatus spatial_dir_apply(FjbRecipe* recipe, const DirPlan& plan, const float* src, ptrdiff_t src_row_bytes,
                           uint32_t components, const float* carrier_b, const float* carrier_g, const float* carrier_r,
                           ptrdiff_t carrier_stride, int width, int height, float* filtered_y, float* filtered_m,
                           float* filtered_c, float* log_raw_b, float* log_raw_g, float* log_raw_r, float* scratch,
                           size_t scratch_bytes, void* stream, FjErrorBuffer* error) {
    if (!filtered_y || !filtered_m || !filtered_c || !log_raw_b || !log_raw_g || !log_raw_r)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    const bool carrier = carrier_b && carrier_g && carrier_r;
    if (!carrier && (!src || !(components == 3 || components == 4)))
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "spatial DIR needs a source image or carrier planes");
    if (recipe->r.params.dir_mode == kDirInactive)
        return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "spatial DIR needs active DIR couplers");
    if (!scratch || scratch_bytes < fjb_spatial_dir_scratch_bytes(width, height))
        return fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "spatial DIR scratch is too small");
    if (reinterpret_cast<uintptr_t>(scratch) % 16 != 0)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "spatial DIR scratch must be 16-byte aligned");
    if (plan.width != width || plan.height != height)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "spatial DIR plan built for another frame size");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t plane = (size_t)width * (size_t)height;
    float* raw[3] = {scratch, scratch + plane, scratch + 2 * plane};
    PixelParams p = recipe->r.params;
    p.src = reinterpret_cast<const char*>(src);
    p.src_row_bytes = src_row_bytes;
    p.components = (int)components;
    p.width = width;
    p.height = height;
    p.carrier_b = carrier_b;
    p.carrier_g = carrier_g;
    p.carrier_r = carrier_r;
    p.carrier_stride = carrier_stride;
    p.dir_src_y = raw[0];
    p.dir_src_m = raw[1];
    p.dir_src_c = raw[2];
    p.dir_src_log_b = log_raw_b;
    p.dir_src_log_g = log_raw_g;
    p.dir_src_log_r = log_raw_r;
    cudaError_t e = launch_pixel_chain(p, carrier ? PixelStage::CarrierToDirSource : PixelStage::SourceToDirSource, s);
    if (e == cudaSuccess) {
        const float* in[3] = {raw[0], raw[1], raw[2]};
        float* out[3] = {filtered_y, filtered_m, filtered_c};
        e = dir_blur_planes(plan, in, out, width, height, scratch, s);
    }
    if (e != cudaSuccess) return cuda_status(e, error, "spatial DIR");
    return ok_status();
}

// The weighted Gaussian components of the plan on three dense width x height planes
// (in -> out, Y, M, C), with the recursion buffers and component planes in `scratch`
// (fjb_spatial_dir_scratch_bytes; its first three planes are not touched).
cudaError_t dir_blur_planes(const DirPlan& plan, const float* const in[3], float* const out[3], int width, int height,
                            float* scratch, cudaStream_t s) {
    const size_t plane = (size_t)width * (size_t)height;
    DirBlurParams bp{};
    bp.width = width;
    bp.height = height;
    {
        const size_t planes_bytes = ((size_t)(3 + 3 * kDirMaxComponents) * plane * sizeof(float) + 255) / 256 * 256;
        char* rec = reinterpret_cast<char*>(scratch) + planes_bytes;
        bp.lines_max = width > height ? width : height;
        const int sw = dir_segments(width), sh = dir_segments(height);
        bp.segs_max = sw > sh ? sw : sh;
        bp.carry = reinterpret_cast<double*>(rec);
        bp.start = bp.carry + (size_t)3 * kDirMaxComponents * bp.lines_max * bp.segs_max * 3;
    }
    bp.count = plan.count;
    for (int k = 0; k < plan.count; ++k) bp.comp[k] = plan.comp[k];
    for (int c = 0; c < 3; ++c) {
        bp.raw[c] = in[c];
        bp.filtered[c] = out[c];
        for (int k = 0; k < kDirMaxComponents; ++k)
            bp.temp[c][k] = scratch + (3 + (size_t)c * kDirMaxComponents + k) * plane;
    }
    return launch_dir_blur(bp, s);
}

} // namespace fjb

extern "C" {

size_t fjb_spatial_dir_scratch_bytes(int32_t width, int32_t height) {
    if (width <= 0 || height <= 0) return 0;
    const size_t planes = (size_t)(3 + 3 * fjb::kDirMaxComponents) * (size_t)width * (size_t)height * sizeof(float);
    return (planes + 255) / 256 * 256 + fjb::dir_recursion_bytes(width, height);
}

FjStatus fjb_spatial_dir_build(FjbRecipe* recipe, const FjSpatialDir* spatial_dir, const float* src,
                               ptrdiff_t src_row_bytes, uint32_t components, const float* carrier_b,
                               const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                               int32_t width, int32_t height, float* filtered_y, float* filtered_m,
                               float* filtered_c, float* log_raw_b, float* log_raw_g, float* log_raw_r,
                               float* scratch, size_t scratch_bytes, void* stream, FjErrorBuffer* error) {
    try {
        if (!recipe || !spatial_dir) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (width <= 0 || height <= 0) {
            write_error(error, "");
            return ok_status();
        }
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        fjb::DirPlan plan;
        std::string why;
        cudaError_t e = cudaSuccess;
        if (!fjb::dir_plan_create(*spatial_dir, width, height, s, plan, why, e)) {
            plan.release();
            if (e != cudaSuccess) return cuda_status(e, error, "spatial DIR plan");
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        }
        FjStatus st = fjb::spatial_dir_apply(recipe, plan, src, src_row_bytes, components, carrier_b, carrier_g,
                                             carrier_r, carrier_stride, width, height, filtered_y, filtered_m,
                                             filtered_c, log_raw_b, log_raw_g, log_raw_r, scratch, scratch_bytes,
                                             stream, error);
        // the plan's device tables must outlive the kernels that read them
        e = cudaStreamSynchronize(s);
        plan.release();
        if (st.category != FJ_STATUS_SUCCESS) return st;
        if (e != cudaSuccess) return cuda_status(e, error, "spatial DIR");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_spatial_dir_build");
    }
}

FjStatus fjb_spatial_dir_blur(const FjSpatialDir* spatial_dir, const float* in_y, const float* in_m,
                              const float* in_c, float* out_y, float* out_m, float* out_c, int32_t width,
                              int32_t height, float* scratch, size_t scratch_bytes, void* stream,
                              FjErrorBuffer* error) {
    try {
        if (!spatial_dir || !in_y || !in_m || !in_c || !out_y || !out_m || !out_c)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (width <= 0 || height <= 0) {
            write_error(error, "");
            return ok_status();
        }
        if (!scratch || scratch_bytes < fjb_spatial_dir_scratch_bytes(width, height))
            return fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "spatial DIR scratch is too small");
        if (reinterpret_cast<uintptr_t>(scratch) % 16 != 0)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "spatial DIR scratch must be 16-byte aligned");
        const size_t plane = (size_t)width * (size_t)height;
        const float* ins[3] = {in_y, in_m, in_c};
        float* outs[3] = {out_y, out_m, out_c};
        const float* region = scratch + 3 * plane;
        for (int c = 0; c < 3; ++c)
            if (ins[c] == outs[c] || (ins[c] >= scratch && ins[c] < region) || (outs[c] >= scratch && outs[c] < region))
                return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "spatial DIR blur planes overlap");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        fjb::DirPlan plan;
        std::string why;
        cudaError_t e = cudaSuccess;
        if (!fjb::dir_plan_create(*spatial_dir, width, height, s, plan, why, e)) {
            plan.release();
            if (e != cudaSuccess) return cuda_status(e, error, "spatial DIR plan");
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        }
        e = fjb::dir_blur_planes(plan, ins, outs, width, height, scratch, s);
        // the plan's device tables must outlive the kernels that read them
        const cudaError_t e2 = cudaStreamSynchronize(s);
        plan.release();
        if (e != cudaSuccess) return cuda_status(e, error, "spatial DIR blur");
        if (e2 != cudaSuccess) return cuda_status(e2, error, "spatial DIR blur");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_spatial_dir_blur");
    }
}

struct FjbDirFilter {
    fjb::DirPlan plan;
};

FjStatus fjb_spatial_dir_filter_create(const FjSpatialDir* spatial_dir, int32_t width, int32_t height, void* stream,
                                       FjbDirFilter** out, FjErrorBuffer* error) {
    try {
        if (!spatial_dir || !out) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        *out = nullptr;
        if (width <= 0 || height <= 0) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "empty frame");
        FjbDirFilter* f = new FjbDirFilter();
        std::string why;
        cudaError_t e = cudaSuccess;
        if (!fjb::dir_plan_create(*spatial_dir, width, height, reinterpret_cast<cudaStream_t>(stream), f->plan, why,
                                  e)) {
            f->plan.release();
            delete f;
            if (e != cudaSuccess) return cuda_status(e, error, "spatial DIR plan");
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        }
        *out = f;
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_spatial_dir_filter_create");
    }
}

FjStatus fjb_spatial_dir_filter_apply(const FjbDirFilter* filter, const float* in_y, const float* in_m,
                                      const float* in_c, float* out_y, float* out_m, float* out_c, float* scratch,
                                      size_t scratch_bytes, void* stream, FjErrorBuffer* error) {
    if (!filter || !in_y || !in_m || !in_c || !out_y || !out_m || !out_c)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    const int width = filter->plan.width, height = filter->plan.height;
    if (!scratch || scratch_bytes < fjb_spatial_dir_scratch_bytes(width, height))
        return fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "spatial DIR scratch is too small");
    if (reinterpret_cast<uintptr_t>(scratch) % 16 != 0)
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "spatial DIR scratch must be 16-byte aligned");
    const size_t plane = (size_t)width * (size_t)height;
    const float* ins[3] = {in_y, in_m, in_c};
    float* outs[3] = {out_y, out_m, out_c};
    const float* region = scratch + 3 * plane;
    for (int c = 0; c < 3; ++c)
        if (ins[c] == outs[c] || (ins[c] >= scratch && ins[c] < region) || (outs[c] >= scratch && outs[c] < region))
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "spatial DIR filter planes overlap");
    const cudaError_t e =
        fjb::dir_blur_planes(filter->plan, ins, outs, width, height, scratch, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e, error, "spatial DIR filter");
    write_error(error, "");
    return ok_status();
}

void fjb_spatial_dir_filter_destroy(FjbDirFilter* filter) {
    if (!filter) return;
    // the filter's device tables may still be read by enqueued work
    cudaDeviceSynchronize();
    filter->plan.release();
    delete filter;
}

FjStatus fjb_recipe_set_spatial_dir_planes(FjbRecipe* recipe, const float* filtered_y, const float* filtered_m,
                                           const float* filtered_c, const float* log_raw_b, const float* log_raw_g,
                                           const float* log_raw_r, FjErrorBuffer* error) {
    if (!recipe) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null recipe");
    fjb::PixelParams& p = recipe->r.params;
    const bool on = filtered_y && filtered_m && filtered_c && log_raw_b && log_raw_g && log_raw_r;
    p.dir_spatial = on ? 1 : 0;
    p.dir_filtered_y = on ? filtered_y : nullptr;
    p.dir_filtered_m = on ? filtered_m : nullptr;
    p.dir_filtered_c = on ? filtered_c : nullptr;
    p.dir_log_raw_b = on ? log_raw_b : nullptr;
    p.dir_log_raw_g = on ? log_raw_g : nullptr;
    p.dir_log_raw_r = on ? log_raw_r : nullptr;
    write_error(error, "");
    return ok_status();
}

FjStatus fjb_dir_boundary_host(const FjDirGaussian* component, int32_t axis_length, double* weights,
                               size_t weights_capacity, int32_t* out_length, int32_t* out_terminal_size,
                               double* terminal, FjErrorBuffer* error) {
    try {
        if (!component || !weights || !out_length || !out_terminal_size || !terminal)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        fjb::DirAxisBoundary b;
        std::string why;
        if (!fjb::dir_axis_boundary(*component, axis_length, b, why))
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        if (b.weights.size() > weights_capacity)
            return fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "boundary weights exceed the buffer");
        for (size_t i = 0; i < b.weights.size(); ++i) weights[i] = b.weights[i];
        for (int i = 0; i < 9; ++i) terminal[i] = b.terminal[i];
        *out_length = b.length;
        *out_terminal_size = b.terminal_size;
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_dir_boundary_host");
    }
}

} // extern "C"
