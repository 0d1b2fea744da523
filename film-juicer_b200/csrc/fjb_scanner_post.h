// fjb_scanner_post.h -- scanner post effects (glare, lens blur, unsharp) on planes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/juicer_cuda_api.h"

struct FjbRecipe;

namespace fjb {

constexpr int kMaxGaussianRadius = 2048; // rust/film-juicer-core/src/optics/gaussian.rs:21

// Glare percent plane (dense, width floats per row).
cudaError_t launch_glare(float* out, int width, int height, uint64_t seed, uint32_t medium, int origin_x,
                         int origin_y, float percent, float roughness, cudaStream_t stream);

// Separable Gaussian blur of `count` (1..3) planes in place through as many `tmps`
// (taps w[0..2r], device).
cudaError_t launch_blur_planes(float* const* planes, float* const* tmps, int count, int width, int height,
                               const float* w, int radius, cudaStream_t stream);

// plane <- plane + amount (plane - blur(plane)) for `count` (1..3) planes, through `tmps`.
cudaError_t launch_unsharp_planes(float* const* planes, float* const* tmps, int count, int width, int height,
                                  const float* w, int radius, float amount, cudaStream_t stream);

// Which effects a post-effects record turns on, with their Gaussian taps (host).
struct PostPlan {
    bool active = false;
    bool glare = false;
    float glare_percent = 0.0f, glare_roughness = 0.0f;
    std::vector<float> glare_w, lens_w, unsharp_w; // empty: that blur is off
    int glare_r = 0, lens_r = 0, unsharp_r = 0;
    float unsharp_amount = 0.0f;
    size_t taps() const { return glare_w.size() + lens_w.size() + unsharp_w.size(); }
};
bool post_plan_from(const FjScannerPostEffects& d, PostPlan& plan, std::string& why);

// Glare seed of a frame: FNV-1a over the 8-byte words {recipe hash, frame token,
// source x1, source y1} (src/Cuda/JuicerCudaExecutor.cpp:2416, src/Hash.h:50).
uint64_t glare_seed(uint64_t recipe_hash, uint64_t frame_token, int32_t x1, int32_t y1);

// Floats of scratch for a frame: six planes (linear R, G, B, blur temp, glare, glare
// blur temp) and room for the taps.
size_t post_scratch_floats(int width, int height);
std::vector<float> post_taps(const PostPlan& plan);

// Film-defect effects on the way out: the dust transmittance plane, and with the gate
// output on, weave and gate mask at the encoding.
struct OutputEffects {
    const float* dust = nullptr;
    bool weave = false;
    float weave_dx = 0.0f, weave_dy = 0.0f, weave_cos = 1.0f, weave_sin = 0.0f;
    const float* gate_mask = nullptr;
    int gate_w = 0, gate_h = 0, roi_x = 0, roi_y = 0;
};

// Density planes -> glare -> linear output RGB -> lens blur -> unsharp -> encoded dst.
// `taps` (device) holds post_taps(plan).
FjStatus render_from_density_post(FjbRecipe* recipe, const PostPlan& plan, uint64_t seed, int32_t origin_x,
                                  int32_t origin_y, const float* density_c, const float* density_m,
                                  const float* density_y, const float* src, ptrdiff_t src_row_bytes, float* dst,
                                  ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                  float* scratch, const float* taps, cudaStream_t s, FjErrorBuffer* error,
                                  const OutputEffects& fx = OutputEffects{});

} // namespace fjb
