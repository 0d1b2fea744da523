// fjb_api_scanner_post.cpp -- scanner post effects: planning, glare seed, Gaussian taps
// and the extern "C" stage entry that scans density planes through them.
//
// Follows the reference's schedule for a frame whose scanner post effects are active
// (src/Cuda/JuicerCudaExecutor.cpp:2384-2500 scan_print_output,
// src/Cuda/Scan/JuicerCudaScanPipeline.cu:2586-2878): glare percent plane (+ its blur),
// scan of the density planes to linear output RGB with the glare added in XYZ, lens
// blur of each plane, unsharp mask of each plane, output encoding.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "fjb_dir.h"
#include "fjb_internal.h"
#include "fjb_recipe.h"
#include "fjb_scanner_post.h"
#include "fjb_schedule.h"

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

namespace fjb {

namespace {

bool taps_for(int radius, float sigma, std::vector<float>& w, const char* what, std::string& why) {
    if (radius < 1 || radius > kMaxGaussianRadius || !(sigma > 0.0f) || !std::isfinite(sigma)) {
        why = std::string("scanner post effects: ") + what + " Gaussian radius outside 1..2048 or sigma not positive";
        return false;
    }
    w = gaussian_taps(radius, sigma);
    return !w.empty();
}

} // namespace

// The reference decodes the record at native/juicer_cuda_descriptors.cpp:538-566 (active
// when its hash is non-zero), builds the kernels at src/ProcessRoot.cpp:3121-3156 and
// gates each effect at src/Cuda/Scan/JuicerCudaScanPipeline.cu:2626-2630, :2803-2813.
bool post_plan_from(const FjScannerPostEffects& d, PostPlan& plan, std::string& why) {
    plan = PostPlan{};
    if ((d.flags & ~FJ_POST_GLARE) != 0) {
        why = "scanner post effects: unknown flags";
        return false;
    }
    plan.active = d.hash != 0;
    if (!plan.active) return true;
    const bool glare_flag = (d.flags & FJ_POST_GLARE) != 0;
    if (d.lens_blur_sigma_px > 0.0f && !taps_for(d.lens_blur_radius, d.lens_blur_sigma_px, plan.lens_w, "lens blur", why))
        return false;
    if (d.unsharp_sigma_px > 0.0f && !taps_for(d.unsharp_radius, d.unsharp_sigma_px, plan.unsharp_w, "unsharp", why))
        return false;
    if (glare_flag && d.glare_blur_sigma_px > 0.0f &&
        !taps_for(d.glare_blur_radius, d.glare_blur_sigma_px, plan.glare_w, "glare blur", why))
        return false;
    plan.lens_r = plan.lens_w.empty() ? 0 : d.lens_blur_radius;
    plan.glare_r = plan.glare_w.empty() ? 0 : d.glare_blur_radius;
    plan.glare = std::isfinite(d.glare_percent) && d.glare_percent > 0.0f && std::isfinite(d.glare_roughness);
    plan.glare_percent = d.glare_percent;
    plan.glare_roughness = d.glare_roughness;
    const bool unsharp = !plan.unsharp_w.empty() && std::isfinite(d.unsharp_amount) && d.unsharp_amount > 0.0f;
    plan.unsharp_r = unsharp ? d.unsharp_radius : 0;
    if (!unsharp) plan.unsharp_w.clear();
    plan.unsharp_amount = d.unsharp_amount;
    return true;
}

uint64_t glare_seed(uint64_t recipe_hash, uint64_t frame_token, int32_t x1, int32_t y1) {
    uint64_t h = 0xcbf29ce484222325ULL;
    const uint64_t words[4] = {recipe_hash, frame_token, (uint64_t)(int64_t)x1, (uint64_t)(int64_t)y1};
    for (uint64_t w : words)
        for (int b = 0; b < 8; ++b) {
            h ^= (w >> (8 * b)) & 0xffu;
            h *= 0x100000001b3ULL;
        }
    return h;
}

size_t post_scratch_floats(int width, int height) {
    const size_t plane = ((size_t)width * (size_t)height + 63) / 64 * 64;
    return 6 * plane + (size_t)3 * (2 * kMaxGaussianRadius + 1 + 63) / 64 * 64;
}

// Scratch: linear R, G, B planes, blur temp, glare, glare blur temp, then the taps.
// After the scan, the last three planes serve as the temps of the three-plane blurs.
// `taps` (device) holds glare, lens and unsharp taps back to back, as in the plan.
FjStatus render_from_density_post(FjbRecipe* recipe, const PostPlan& plan, uint64_t seed, int32_t origin_x,
                                  int32_t origin_y, const float* density_c, const float* density_m,
                                  const float* density_y, const float* src, ptrdiff_t src_row_bytes, float* dst,
                                  ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                  float* scratch, const float* taps, cudaStream_t s, FjErrorBuffer* error,
                                  const OutputEffects& fx) {
    const size_t plane = ((size_t)width * (size_t)height + 63) / 64 * 64;
    float* lin[3] = {scratch, scratch + plane, scratch + 2 * plane};
    float* tmp = scratch + 3 * plane;
    float* glare = scratch + 4 * plane;
    float* blurred = scratch + 5 * plane;
    const float* glare_w = taps;
    const float* lens_w = glare_w + plan.glare_w.size();
    const float* unsharp_w = lens_w + plan.lens_w.size();
    PixelParams p = recipe->r.params;
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
    p.lin_r = lin[0];
    p.lin_g = lin[1];
    p.lin_b = lin[2];
    p.scan_glare = nullptr;
    p.film_dust = fx.dust;
    cudaError_t e = cudaSuccess;
    if (plan.glare) {
        const uint32_t medium = p.scan_medium_negative ? 0u : 1u;
        e = launch_glare(glare, width, height, seed, medium, origin_x, origin_y, plan.glare_percent,
                         plan.glare_roughness, s);
        if (e == cudaSuccess && plan.glare_r > 0) e = launch_blur_planes(&glare, &blurred, 1, width, height, glare_w, plan.glare_r, s);
        p.scan_glare = glare;
    }
    if (e == cudaSuccess && p.route == kRoutePrint && p.print_form != kPrintFp32 && !p.print_done) {
        // the tensor-core form hands the spectral integral to the FP32 epilogue in planes
        e = recipe->r.ensure_tc_raw((size_t)width * (size_t)height);
        p.tc_raw = recipe->r.tc_raw;
    }
    if (e == cudaSuccess) e = launch_pixel_chain(p, PixelStage::DensityToLinearRgb, s);
    // the glare planes are free once the scan has added the glare: the three planes blur
    // together through tmp, glare and the glare blur temp
    float* tmps[3] = {tmp, glare, blurred};
    if (e == cudaSuccess && plan.lens_r > 0) e = launch_blur_planes(lin, tmps, 3, width, height, lens_w, plan.lens_r, s);
    if (e == cudaSuccess && plan.unsharp_r > 0)
        e = launch_unsharp_planes(lin, tmps, 3, width, height, unsharp_w, plan.unsharp_r, plan.unsharp_amount, s);
    p.weave_active = fx.weave ? 1 : 0;
    p.weave_dx = fx.weave_dx;
    p.weave_dy = fx.weave_dy;
    p.weave_cos = fx.weave_cos;
    p.weave_sin = fx.weave_sin;
    p.gate_mask = fx.gate_mask;
    p.gate_w = fx.gate_w;
    p.gate_h = fx.gate_h;
    p.roi_x = fx.roi_x;
    p.roi_y = fx.roi_y;
    if (e == cudaSuccess) e = launch_pixel_chain(p, PixelStage::LinearRgbToOutput, s);
    if (e != cudaSuccess) return cuda_status(e, error, "scanner post effects");
    write_error(error, "");
    return ok_status();
}

// Taps of a plan, in the order render_from_density_post expects them.
std::vector<float> post_taps(const PostPlan& plan) {
    std::vector<float> t;
    t.insert(t.end(), plan.glare_w.begin(), plan.glare_w.end());
    t.insert(t.end(), plan.lens_w.begin(), plan.lens_w.end());
    t.insert(t.end(), plan.unsharp_w.begin(), plan.unsharp_w.end());
    return t;
}

} // namespace fjb

extern "C" {

FjStatus fjb_gaussian_kernel_host(int32_t radius, float sigma_px, float* weights, size_t count,
                                  FjErrorBuffer* error) {
    try {
        if (!weights) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (radius < 1 || radius > fjb::kMaxGaussianRadius)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "Gaussian radius outside 1..2048");
        if (!(sigma_px > 0.0f) || !std::isfinite(sigma_px))
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "Gaussian sigma not positive and finite");
        if (count < (size_t)(2 * radius + 1))
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "weights buffer shorter than 2 radius + 1");
        const std::vector<float> w = fjb::gaussian_taps(radius, sigma_px);
        std::memcpy(weights, w.data(), w.size() * sizeof(float));
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_gaussian_kernel_host");
    }
}

uint64_t fjb_glare_seed(uint64_t recipe_hash, uint64_t frame_token, int32_t source_x1, int32_t source_y1) {
    return fjb::glare_seed(recipe_hash, frame_token, source_x1, source_y1);
}

size_t fjb_scanner_post_scratch_bytes(int32_t width, int32_t height) {
    if (width <= 0 || height <= 0) return 0;
    return fjb::post_scratch_floats(width, height) * sizeof(float);
}

FjStatus fjb_render_from_density_post(FjbRecipe* recipe, const FjScannerPostEffects* post, uint64_t glare_seed,
                                      int32_t glare_origin_x, int32_t glare_origin_y, const float* density_c,
                                      const float* density_m, const float* density_y, const float* src,
                                      ptrdiff_t src_row_bytes, float* dst, ptrdiff_t dst_row_bytes, int32_t width,
                                      int32_t height, uint32_t components, float* scratch, size_t scratch_bytes,
                                      void* stream, FjErrorBuffer* error) {
    try {
        if (!recipe || !post || !density_c || !density_m || !density_y || !dst || !scratch)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (!(components == FJ_COMPONENTS_RGB || components == FJ_COMPONENTS_RGBA) || width < 0 || height < 0)
            return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unsupported image geometry");
        if (components == FJ_COMPONENTS_RGBA && !src)
            return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "RGBA output needs the source for alpha");
        if (width == 0 || height == 0) {
            write_error(error, "");
            return ok_status();
        }
        if (scratch_bytes < fjb_scanner_post_scratch_bytes(width, height))
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "scanner post scratch too small");
        fjb::PostPlan plan;
        std::string why;
        if (!fjb::post_plan_from(*post, plan, why)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        float* taps = scratch + fjb::post_scratch_floats(width, height) -
                      (size_t)3 * (2 * fjb::kMaxGaussianRadius + 1 + 63) / 64 * 64;
        const std::vector<float> t = fjb::post_taps(plan);
        // pageable source: the copy is staged before the call returns
        if (!t.empty()) {
            cudaError_t e = cudaMemcpyAsync(taps, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) return cuda_status(e, error, "scanner post taps");
        }
        return fjb::render_from_density_post(recipe, plan, glare_seed, glare_origin_x, glare_origin_y, density_c,
                                             density_m, density_y, src, src_row_bytes, dst, dst_row_bytes, width,
                                             height, components, scratch, taps, s, error);
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_render_from_density_post");
    }
}

} // extern "C"
