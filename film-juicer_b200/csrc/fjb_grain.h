// fjb_grain.h -- density-space visual grain (device side).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fjb {

constexpr int kGrainMaxRadius = 75; // the host plan caps every grain Gaussian at 75

// Per-frame values derived once on the device (breathing and clump fields).
struct GrainFrameUniforms {
    int breathing_active;
    float breathing_t;
    uint64_t breathing_seed_a, breathing_seed_b;
    float breathing_cell_small_px, breathing_cell_large_px;
    float breathing_drift_x, breathing_drift_y, breathing_roll_y;
    float breathing_mix;
    int clump_active;
    float clump_cell_px, clump_roll_y;
    uint64_t clump_static_seed;
    float clump_rms_norm, clump_mu, clump_sigma;
};

// Everything the grain kernels read about one frame (one pass of one scale overrides
// the seeds and the particle table). Curves: the capture density curve of each CMY
// channel (the layer interpolation axis) and the nine [layer][channel] layer curves.
struct GrainFrame {
    int origin_x, origin_y;
    int positive_film;
    int sublayers;
    int n_sublayers;
    uint64_t seed_base, seed_base_next;
    int64_t frame_index;
    float time_alpha;
    uint64_t session_seed, clip_token;
    // static blue noise and Wang tiles
    const uint8_t* stbn;
    int stbn_w, stbn_h, stbn_frames;
    int stbn_offset_x, stbn_offset_y, stbn_frame;
    const uint8_t* wang_tiles;
    const uint8_t* wang_lut;
    int wang_w, wang_h, wang_count, wang_colors;
    float wang_cell_mm;
    // temporal fields
    int breathing_period_frames;
    float breathing_amplitude, breathing_cell_um_small, breathing_cell_um_large, breathing_mix,
        breathing_drift_um_per_frame;
    float pixel_size_um;
    int pitch_px;
    float micro_structure[2];
    float clump_temporal_mix;
    int clump_morph_period_frames;
    // particle model
    float density_min[3], uniformity[3], density_max[3], n_particles[3], od_particle[3];
    float density_min_layers[3][3], density_max_layers[3][3], n_particles_layers[3][3], od_particle_layers[3][3];
    const float* base_curve[3]; // density values of the capture curve, per CMY channel
    int base_curve_n[3];
    int axis_finite[3];
    float axis_block_prefix_max[3][16];
    const float* layer_curve[3][3];
    GrainFrameUniforms* uniforms;
};

enum GrainSampleMode : int { kGrainSimple = 0, kGrainLayer = 1, kGrainTriplet = 2 };

// What the sample kernel does with its value before storing it:
//   store: out = value (a layer plane that a dye-cloud blur reads next);
//   accumulate: out = sanitize((init ? 0 : out) + value);
//   then optionally forms the scale's delta against the density plane.
struct GrainSampleEpilogue {
    int accumulate;
    int init;
    int form_delta;
    float density_bias;
};

struct GrainBlurTaps {
    int radius;
    float w[2 * kGrainMaxRadius + 1];
};

// Vertical-pass epilogue (see fjb_grain.cu).
struct GrainVerticalEpilogue {
    int weighted;
    float weight;
    int init;
    const float* density; // non-null: form the delta (unweighted pass only)
    long long density_stride;
    float density_bias;
    int apply_gain;
    float gain;
};

struct GrainPlane {
    float* p;
    long long stride;
};

cudaError_t launch_grain_uniforms(const GrainFrame& f, cudaStream_t s);
cudaError_t launch_grain_sample(const GrainFrame& f, int mode, int channel, int layer, const float* density,
                                long long density_stride, GrainPlane out, const GrainSampleEpilogue& ep, int width,
                                int height, cudaStream_t s);
cudaError_t launch_grain_blur_rows(const float* in, long long in_stride, float* out, long long out_stride,
                                   const GrainBlurTaps& taps, int width, int height, cudaStream_t s);
cudaError_t launch_grain_blur_columns(const float* in, long long in_stride, GrainPlane out,
                                      const GrainBlurTaps& taps, const GrainVerticalEpilogue& ep, int width,
                                      int height, cudaStream_t s);
// dst = sanitize((init ? 0 : dst) + weight * src), then optionally x gain.
cudaError_t launch_grain_accumulate_weighted(GrainPlane dst, const float* src, long long src_stride, float weight,
                                             int init, int apply_gain, float gain, int width, int height,
                                             cudaStream_t s);
cudaError_t launch_grain_clear(GrainPlane dst, int width, int height, cudaStream_t s);
// density = sanitize(fma(scale, delta', add_mean ? density : 0)) with delta' the delta
// (independent) or the shared/independent mix when `shared` is non-null.
cudaError_t launch_grain_finish(float* density, long long density_stride, const float* delta, long long delta_stride,
                                const float* shared, float shared_weight, float independent_weight, float amplitude,
                                float scale, int add_mean, int width, int height, cudaStream_t s);
// debug: all three planes = offset + mean(c, m, y) * scale
cudaError_t launch_grain_debug_average(float* c, float* m, float* y, long long stride, float offset, float scale,
                                       int width, int height, cudaStream_t s);

} // namespace fjb
