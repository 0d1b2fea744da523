// fjb_api_grain.cpp -- extern "C" entry points of the visual grain stage.
//
// The pass schedule restates src/Cuda/Scan/JuicerCudaScanPipeline.cu:3141-3740
// (juicer_cuda_apply_visual_grain) with the payload packing of
// src/Cuda/JuicerCudaFilmPayloads.cpp:212-240 and :384-495; kernels in fjb_grain.cu.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "fjb_dir.h"
#include "fjb_grain.h"
#include "fjb_recipe.h"
#include "fjb_schedule.h"

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

struct FjbNoise {
    uint8_t* stbn = nullptr;
    uint8_t* wang_tiles = nullptr;
    uint8_t* wang_lut = nullptr;
    int stbn_w = 0, stbn_h = 0, stbn_frames = 0;
    int wang_w = 0, wang_h = 0, wang_count = 0, wang_colors = 0;
    void release() {
        for (void* p : {(void*)stbn, (void*)wang_tiles, (void*)wang_lut})
            if (p) cudaFree(p);
        stbn = wang_tiles = wang_lut = nullptr;
    }
};

namespace {

constexpr size_t kUniformBytes = 256;
constexpr int kGrainPlanes = 5; // row-blur temp, scale work, delta accumulator, layer work, shared delta

constexpr uint64_t kSaltFine = 0xA24BAED4963EE407ULL;
constexpr uint64_t kSaltMid = 0x9F6C1E6B2C4D7A13ULL;
constexpr uint64_t kSaltCoarse = 0x3C79AC492BA7B653ULL;
constexpr uint64_t kSaltShared = 0x7E8A1B9D3F2C65A1ULL;

// FNV-1a over the little-endian bytes of each value (src/Hash.h:50-56).
uint64_t fnv_u64s(std::initializer_list<uint64_t> values) {
    uint64_t h = 0xcbf29ce484222325ULL;
    for (uint64_t v : values)
        for (int i = 0; i < 8; ++i) {
            h ^= (v >> (8 * i)) & 0xFFu;
            h *= 0x100000001b3ULL;
        }
    return h;
}

int stbn_offset(uint64_t session_seed, int dimension, uint64_t salt) {
    if (dimension <= 0) return 0;
    return (int)(fnv_u64s({session_seed, salt}) % (uint64_t)dimension);
}

int stbn_frame_index(int64_t frame, int count, uint64_t session_seed) {
    if (count <= 0) return 0;
    const int64_t phase = (int64_t)(session_seed % (uint64_t)count);
    int f = (int)((frame + phase) % count);
    return f < 0 ? f + count : f;
}

bool finite_positive(float v) { return std::isfinite(v) && v > 0.0f; }

struct Taps {
    fjb::GrainBlurTaps t{};
    uint64_t hash = 0;
    bool active() const { return t.radius > 0; }
};

bool make_taps(const FjGrainGaussian& g, Taps& out, std::string& why) {
    out = Taps{};
    if (g.radius <= 0) return true;
    if (g.radius > fjb::kGrainMaxRadius || !finite_positive(g.sigma_px)) {
        why = "grain Gaussian radius outside 1..75 or sigma not positive";
        return false;
    }
    const std::vector<float> w = fjb::gaussian_taps(g.radius, g.sigma_px);
    if ((int)w.size() != 2 * g.radius + 1) {
        why = "grain Gaussian taps";
        return false;
    }
    out.t.radius = g.radius;
    for (size_t i = 0; i < w.size(); ++i) out.t.w[i] = w[i];
    out.hash = g.hash;
    return true;
}

struct Schedule {
    const FjVisualGrain* g;
    fjb::GrainFrame base;
    Taps corr[3];
    Taps dye[3][3];
    int width, height;
    fjb::GrainPlane temp, scale, accum, layer, shared;
    cudaStream_t s;

    // One particle-size scale of one channel into `target` (src JuicerCudaScanPipeline.cu
    // generate_scale): sample, dye-cloud blur, delta, correlation blur, weighted sum.
    cudaError_t scale_pass(const fjb::GrainFrame& frame, const float* density, long long dstride, int ch,
                           uint64_t salt, float factor, const Taps& corr, bool apply_corr, float weight, bool init,
                           fjb::GrainPlane target, bool apply_gain, float gain) {
        fjb::GrainFrame f = frame;
        f.seed_base ^= salt;
        f.seed_base_next ^= salt;
        if (!(std::isfinite(factor) && factor > 0.0f)) return cudaErrorInvalidValue;
        for (int c = 0; c < 3; ++c) {
            f.n_particles[c] = frame.n_particles[c] / factor;
            f.od_particle[c] = frame.od_particle[c] * factor;
            for (int l = 0; l < 3; ++l) {
                f.n_particles_layers[l][c] = frame.n_particles_layers[l][c] / factor;
                f.od_particle_layers[l][c] = frame.od_particle_layers[l][c] * factor;
            }
        }
        const float bias = -frame.density_min[ch];
        cudaError_t e = cudaSuccess;
        bool delta_formed = false;
        if (f.sublayers) {
            const Taps& d0 = dye[0][ch];
            const Taps& d1 = dye[1][ch];
            const Taps& d2 = dye[2][ch];
            // one shared blur when the three layers' dye clouds are the same prepared
            // Gaussian (equal identity), or when none of them blurs
            const bool all_zero = !d0.active() && !d1.active() && !d2.active();
            const bool same = d0.t.radius == d1.t.radius && d0.t.radius == d2.t.radius &&
                              (all_zero || (d0.hash == d1.hash && d0.hash == d2.hash));
            if (same && (d0.active() || all_zero)) {
                if (d0.active()) {
                    const fjb::GrainSampleEpilogue ep{0, 0, 0, 0.0f};
                    if ((e = fjb::launch_grain_sample(f, fjb::kGrainTriplet, ch, 0, density, dstride, layer, ep, width,
                                                      height, s)) != cudaSuccess)
                        return e;
                    if ((e = fjb::launch_grain_blur_rows(layer.p, layer.stride, temp.p, temp.stride, d0.t, width,
                                                         height, s)) != cudaSuccess)
                        return e;
                    const fjb::GrainVerticalEpilogue vep{0, 0.0f, 1, density, dstride, bias, 0, 1.0f};
                    if ((e = fjb::launch_grain_blur_columns(temp.p, temp.stride, scale, d0.t, vep, width, height,
                                                            s)) != cudaSuccess)
                        return e;
                } else {
                    const fjb::GrainSampleEpilogue ep{1, 1, 1, bias};
                    if ((e = fjb::launch_grain_sample(f, fjb::kGrainTriplet, ch, 0, density, dstride, scale, ep, width,
                                                      height, s)) != cudaSuccess)
                        return e;
                }
                delta_formed = true;
            } else {
                for (int l = 0; l < 3; ++l) {
                    const Taps& d = dye[l][ch];
                    if (d.active()) {
                        const fjb::GrainSampleEpilogue ep{0, 0, 0, 0.0f};
                        if ((e = fjb::launch_grain_sample(f, fjb::kGrainLayer, ch, l, density, dstride, layer, ep,
                                                          width, height, s)) != cudaSuccess)
                            return e;
                        if ((e = fjb::launch_grain_blur_rows(layer.p, layer.stride, temp.p, temp.stride, d.t, width,
                                                             height, s)) != cudaSuccess)
                            return e;
                        const fjb::GrainVerticalEpilogue vep{0,   0.0f, l == 0 ? 1 : 0, l == 2 ? density : nullptr,
                                                             dstride, bias, 0, 1.0f};
                        if ((e = fjb::launch_grain_blur_columns(temp.p, temp.stride, scale, d.t, vep, width, height,
                                                                s)) != cudaSuccess)
                            return e;
                        delta_formed = l == 2;
                    } else {
                        // last unblurred layer forms the delta in the same pass
                        const fjb::GrainSampleEpilogue ep{1, l == 0 ? 1 : 0, l == 2 ? 1 : 0, bias};
                        if ((e = fjb::launch_grain_sample(f, fjb::kGrainLayer, ch, l, density, dstride, scale, ep,
                                                          width, height, s)) != cudaSuccess)
                            return e;
                        if (l == 2) delta_formed = true;
                    }
                }
            }
        } else {
            const fjb::GrainSampleEpilogue ep{0, 0, 1, bias};
            if ((e = fjb::launch_grain_sample(f, fjb::kGrainSimple, ch, 0, density, dstride, scale, ep, width, height,
                                              s)) != cudaSuccess)
                return e;
            delta_formed = true;
        }
        if (!delta_formed) return cudaErrorInvalidValue; // every branch above forms it
        if (apply_corr && corr.active()) {
            if ((e = fjb::launch_grain_blur_rows(scale.p, scale.stride, temp.p, temp.stride, corr.t, width, height,
                                                 s)) != cudaSuccess)
                return e;
            const fjb::GrainVerticalEpilogue vep{1, weight, init ? 1 : 0, nullptr, 0, 0.0f, apply_gain ? 1 : 0, gain};
            return fjb::launch_grain_blur_columns(temp.p, temp.stride, target, corr.t, vep, width, height, s);
        }
        return fjb::launch_grain_accumulate_weighted(target, scale.p, scale.stride, weight, init ? 1 : 0,
                                                     apply_gain ? 1 : 0, gain, width, height, s);
    }

    // All active scales of one channel, gain applied (generate_mix).
    cudaError_t mix(const fjb::GrainFrame& frame, const float* density, long long dstride, int ch,
                    fjb::GrainPlane target) {
        const float wf = g->size_mix_weights[0], wm = g->size_mix_weights[1], wc = g->size_mix_weights[2];
        const float sms = g->size_mix_scale;
        const float mid_factor = std::sqrt(sms);
        struct Pass {
            bool on;
            uint64_t salt;
            float factor;
            const Taps* corr;
            bool apply;
            float weight;
        } passes[3] = {{wf > 0.0f, kSaltFine, 1.0f, &corr[0], corr[0].active(), wf},
                       {wm > 0.0f, kSaltMid, mid_factor, &corr[1], true, wm},
                       {wc > 0.0f, kSaltCoarse, sms, &corr[2], true, wc}};
        int last = -1;
        for (int i = 0; i < 3; ++i)
            if (passes[i].on) last = i;
        if (last < 0) {
            // no scale carries weight: the accumulator is the gain-scaled zero plane
            return fjb::launch_grain_clear(target, width, height, s);
        }
        bool init = true;
        for (int i = 0; i < 3; ++i) {
            if (!passes[i].on) continue;
            cudaError_t e = scale_pass(frame, density, dstride, ch, passes[i].salt, passes[i].factor, *passes[i].corr,
                                       passes[i].apply, passes[i].weight, init, target, i == last, g->size_mix_gain);
            if (e != cudaSuccess) return e;
            init = false;
        }
        return cudaSuccess;
    }
};

bool validate(const FjVisualGrain& g, const fjb::Recipe& r, std::string& why) {
    const bool sub = (g.flags & FJ_GRAIN_SUBLAYERS) != 0;
    for (int c = 0; c < 3; ++c) {
        if (!std::isfinite(g.particle_density_min_cmy[c]) || !finite_positive(g.density_max_cmy[c]) ||
            !finite_positive(g.n_particles_cmy[c]) || !finite_positive(g.od_particle_cmy[c])) {
            why = "grain particle model of a channel is not finite and positive";
            return false;
        }
        if (!sub) continue;
        for (int l = 0; l < 3; ++l)
            if (!std::isfinite(g.density_min_layers[l][c]) || !finite_positive(g.density_max_layers[l][c]) ||
                !finite_positive(g.n_particles_layers[l][c]) || !finite_positive(g.od_particle_layers[l][c])) {
                why = "grain sublayer particle model is not finite and positive";
                return false;
            }
    }
    if (sub && (!r.layer_curves || r.layer_n != r.params.film_curve[0].n)) {
        why = "grain sublayers need the recipe's nine density-layer curves";
        return false;
    }
    const float wf = g.size_mix_weights[0], wm = g.size_mix_weights[1], wc = g.size_mix_weights[2];
    if (!std::isfinite(wf) || !std::isfinite(wm) || !std::isfinite(wc) || wf < 0.0f || wm < 0.0f || wc < 0.0f ||
        std::fabs((wf + wm + wc) - 1.0f) > 1e-5f || !std::isfinite(g.size_mix_scale) || !(g.size_mix_scale >= 1.0f) ||
        !finite_positive(g.size_mix_gain) || !std::isfinite(g.amplitude) || g.amplitude < 0.0f) {
        why = "grain size mix weights, scale, gain or amplitude out of range";
        return false;
    }
    if ((wm > 0.0f && g.correlation[1].radius <= 0) || (wc > 0.0f && g.correlation[2].radius <= 0)) {
        why = "grain mid/coarse scale without its correlation Gaussian";
        return false;
    }
    if (!std::isfinite(g.chroma_mix) || g.chroma_mix < 0.0f || g.chroma_mix > 1.0f ||
        !std::isfinite(g.chroma_shared_weight) || g.chroma_shared_weight < 0.0f ||
        !std::isfinite(g.chroma_independent_weight) || g.chroma_independent_weight < 0.0f ||
        g.debug_view > FJ_GRAIN_DEBUG_MEAN_DENSITY) {
        why = "grain chroma weights or debug view out of range";
        return false;
    }
    return true;
}

} // namespace

extern "C" FjStatus fjb_noise_create(const FjStaticNoise* noise, void* stream, FjbNoise** out, FjErrorBuffer* error) {
    if (!noise || !out) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    *out = nullptr;
    try {
        const size_t stbn_bytes = (size_t)(noise->stbn_width > 0 ? noise->stbn_width : 0) *
                                  (size_t)(noise->stbn_height > 0 ? noise->stbn_height : 0) *
                                  (size_t)(noise->stbn_frames > 0 ? noise->stbn_frames : 0);
        const size_t wang_bytes = (size_t)(noise->wang_width > 0 ? noise->wang_width : 0) *
                                  (size_t)(noise->wang_height > 0 ? noise->wang_height : 0) * noise->wang_tile_count;
        const size_t colors = noise->wang_colors > 0 ? (size_t)noise->wang_colors : 0;
        const size_t lut_bytes = colors * colors * colors * colors;
        if (stbn_bytes == 0 || !noise->stbn.data || noise->stbn.count != stbn_bytes)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "static blue noise must hold w*h*frames bytes");
        if (wang_bytes == 0 || !noise->wang_tiles.data || noise->wang_tiles.count != wang_bytes || lut_bytes == 0 ||
            !noise->wang_lut.data || noise->wang_lut.count != lut_bytes || noise->wang_tile_count > 255)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "Wang tiles or their colour table are malformed");
        FjbNoise* n = new FjbNoise();
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        cudaError_t e = cudaMalloc(&n->stbn, stbn_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&n->wang_tiles, wang_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&n->wang_lut, lut_bytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(n->stbn, noise->stbn.data, stbn_bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(n->wang_tiles, noise->wang_tiles.data, wang_bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(n->wang_lut, noise->wang_lut.data, lut_bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            n->release();
            delete n;
            return cuda_status(e, error, "static noise upload");
        }
        n->stbn_w = noise->stbn_width;
        n->stbn_h = noise->stbn_height;
        n->stbn_frames = noise->stbn_frames;
        n->wang_w = noise->wang_width;
        n->wang_h = noise->wang_height;
        n->wang_count = (int)noise->wang_tile_count;
        n->wang_colors = noise->wang_colors;
        *out = n;
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "unexpected exception in fjb_noise_create");
    }
}

extern "C" FjStatus fjb_noise_destroy(FjbNoise* noise, FjErrorBuffer* error) {
    if (noise) {
        noise->release();
        delete noise;
    }
    write_error(error, "");
    return ok_status();
}

extern "C" size_t fjb_visual_grain_scratch_bytes(int32_t width, int32_t height) {
    if (width <= 0 || height <= 0) return kUniformBytes;
    return kUniformBytes + (size_t)kGrainPlanes * (size_t)width * (size_t)height * sizeof(float);
}

extern "C" FjStatus fjb_visual_grain(FjbRecipe* recipe, const FjVisualGrain* grain, const FjbNoise* noise,
                                     float* density_c, float* density_m, float* density_y, ptrdiff_t stride,
                                     int32_t width, int32_t height, float* scratch, size_t scratch_bytes,
                                     void* stream, FjErrorBuffer* error) {
    try {
        if (!recipe || !grain || !density_c || !density_m || !density_y)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if ((grain->flags & FJ_GRAIN_ACTIVE) == 0) {
            write_error(error, "");
            return ok_status();
        }
        if (width <= 0 || height <= 0 || stride < width)
            return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "grain frame extent or stride");
        if (!scratch || scratch_bytes < fjb_visual_grain_scratch_bytes(width, height))
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "grain scratch smaller than fjb_visual_grain_scratch_bytes");
        if (reinterpret_cast<uintptr_t>(scratch) % 16 != 0)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "grain scratch must be 16-byte aligned");
        const fjb::Recipe& r = recipe->r;
        std::string why;
        if (!validate(*grain, r, why)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);

        Schedule sc{};
        sc.g = grain;
        sc.width = width;
        sc.height = height;
        sc.s = reinterpret_cast<cudaStream_t>(stream);
        for (int i = 0; i < 3; ++i)
            if (!make_taps(grain->correlation[i], sc.corr[i], why)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        const bool sub = (grain->flags & FJ_GRAIN_SUBLAYERS) != 0;
        for (int l = 0; l < 3; ++l)
            for (int c = 0; c < 3; ++c)
                if (sub && !make_taps(grain->dye_cloud[l][c], sc.dye[l][c], why))
                    return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);

        fjb::GrainFrame& f = sc.base;
        std::memset(&f, 0, sizeof(f));
        f.origin_x = grain->render_extent.x;
        f.origin_y = grain->render_extent.y;
        f.positive_film = r.positive_film ? 1 : 0;
        f.sublayers = sub ? 1 : 0;
        f.n_sublayers = (int)grain->sublayer_count;
        f.seed_base = grain->seed_base;
        f.seed_base_next = grain->seed_base_next;
        f.frame_index = grain->frame0;
        f.time_alpha = grain->frame_alpha;
        f.session_seed = grain->session_seed;
        f.clip_token = grain->clip_token;
        if (noise) {
            f.stbn = noise->stbn;
            f.stbn_w = noise->stbn_w;
            f.stbn_h = noise->stbn_h;
            f.stbn_frames = noise->stbn_frames;
            f.wang_tiles = noise->wang_tiles;
            f.wang_lut = noise->wang_lut;
            f.wang_w = noise->wang_w;
            f.wang_h = noise->wang_h;
            f.wang_count = noise->wang_count;
            f.wang_colors = noise->wang_colors;
        }
        f.stbn_offset_x = stbn_offset(grain->session_seed, f.stbn_w, 0xA5u);
        f.stbn_offset_y = stbn_offset(grain->session_seed, f.stbn_h, 0x5Au);
        f.stbn_frame = stbn_frame_index(grain->frame0, f.stbn_frames, grain->session_seed);
        f.wang_cell_mm = grain->wang_cell_mm;
        f.breathing_period_frames = grain->breathing_period_frames;
        f.breathing_amplitude = grain->breathing_amplitude;
        f.breathing_cell_um_small = grain->breathing_cell_um_small;
        f.breathing_cell_um_large = grain->breathing_cell_um_large;
        f.breathing_mix = grain->breathing_mix;
        f.breathing_drift_um_per_frame = grain->breathing_drift_um_per_frame;
        f.pixel_size_um = grain->pixel_size_um;
        f.pitch_px = grain->pitch_px;
        f.micro_structure[0] = grain->micro_structure[0];
        f.micro_structure[1] = grain->micro_structure[1];
        f.clump_temporal_mix = grain->clump_temporal_mix;
        f.clump_morph_period_frames = grain->clump_morph_period_frames;
        for (int c = 0; c < 3; ++c) {
            f.density_min[c] = grain->particle_density_min_cmy[c];
            f.uniformity[c] = grain->uniformity_cmy[c];
            f.density_max[c] = grain->density_max_cmy[c];
            f.n_particles[c] = grain->n_particles_cmy[c];
            f.od_particle[c] = grain->od_particle_cmy[c];
            for (int l = 0; l < 3; ++l) {
                f.density_min_layers[l][c] = grain->density_min_layers[l][c];
                f.density_max_layers[l][c] = grain->density_max_layers[l][c];
                f.n_particles_layers[l][c] = grain->n_particles_layers[l][c];
                f.od_particle_layers[l][c] = grain->od_particle_layers[l][c];
            }
            if (sub) {
                // capture density curve of channel c (C <- red-exposed layer): blob order is B, G, R
                const fjb::CurveRef& cr = r.params.film_curve[2 - c];
                f.base_curve[c] = r.curves + cr.y;
                f.base_curve_n[c] = cr.n;
                f.axis_finite[c] = (grain->flags & (FJ_GRAIN_AXIS_FINITE_C << c)) != 0 ? 1 : 0;
                for (int b = 0; b < 16; ++b) f.axis_block_prefix_max[c][b] = grain->layer_axis_block_prefix_max[c][b];
                for (int l = 0; l < 3; ++l) f.layer_curve[l][c] = r.layer_curves + (size_t)(l * 3 + c) * r.layer_n;
            }
        }
        f.uniforms = reinterpret_cast<fjb::GrainFrameUniforms*>(scratch);

        const size_t plane = (size_t)width * (size_t)height;
        float* planes = scratch + kUniformBytes / sizeof(float);
        auto P = [&](int i) { return fjb::GrainPlane{planes + (size_t)i * plane, (long long)width}; };
        sc.temp = P(0);
        sc.scale = P(1);
        sc.accum = P(2);
        sc.layer = P(3);
        sc.shared = P(4);
        float* density[3] = {density_c, density_m, density_y};
        const long long ds = (long long)stride;
        cudaError_t e = cudaSuccess;
        const uint32_t debug = grain->debug_view;

        if (debug == FJ_GRAIN_DEBUG_MEAN_DENSITY) {
            e = fjb::launch_grain_debug_average(density_c, density_m, density_y, ds, 0.0f, grain->debug_scale * 4.0f,
                                                width, height, sc.s);
            if (e != cudaSuccess) return cuda_status(e, error, "grain debug average");
            write_error(error, "");
            return ok_status();
        }
        if ((e = fjb::launch_grain_uniforms(f, sc.s)) != cudaSuccess) return cuda_status(e, error, "grain uniforms");

        if (debug >= FJ_GRAIN_DEBUG_DELTA_FINE && debug <= FJ_GRAIN_DEBUG_DELTA_COARSE_RAW) {
            const bool coarse = debug == FJ_GRAIN_DEBUG_DELTA_COARSE || debug == FJ_GRAIN_DEBUG_DELTA_COARSE_RAW;
            const bool raw = debug == FJ_GRAIN_DEBUG_DELTA_FINE_RAW || debug == FJ_GRAIN_DEBUG_DELTA_COARSE_RAW;
            for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
                if (!coarse || grain->size_mix_weights[2] > 0.0f) {
                    const Taps& corr = coarse ? sc.corr[2] : sc.corr[0];
                    e = sc.scale_pass(f, density[c], ds, c, coarse ? kSaltCoarse : kSaltFine,
                                      coarse ? grain->size_mix_scale : 1.0f, corr, !raw && corr.active(), 1.0f, true,
                                      sc.accum, false, 1.0f);
                } else {
                    e = fjb::launch_grain_clear(sc.accum, width, height, sc.s);
                }
                if (e == cudaSuccess)
                    e = fjb::launch_grain_finish(density[c], ds, sc.accum.p, sc.accum.stride, nullptr, 0.0f, 0.0f,
                                                 0.0f, grain->amplitude, 0, width, height, sc.s);
            }
        } else {
            const bool shared_chroma = (debug == FJ_GRAIN_DEBUG_OFF || debug == FJ_GRAIN_DEBUG_DELTA_MIX) &&
                                       grain->chroma_mix < 0.999f && grain->chroma_shared_weight > 0.0f;
            if (shared_chroma) {
                fjb::GrainFrame sf = f;
                sf.seed_base ^= kSaltShared;
                sf.seed_base_next ^= kSaltShared;
                e = sc.mix(sf, density_m, ds, 1, sc.shared);
            }
            for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
                const bool independent = grain->chroma_independent_weight > 0.0f || !shared_chroma;
                if (independent) e = sc.mix(f, density[c], ds, c, sc.accum);
                if (e == cudaSuccess)
                    e = fjb::launch_grain_finish(density[c], ds, sc.accum.p, sc.accum.stride,
                                                 shared_chroma ? sc.shared.p : nullptr, grain->chroma_shared_weight,
                                                 grain->chroma_independent_weight, grain->amplitude,
                                                 shared_chroma ? 1.0f : grain->amplitude,
                                                 debug == FJ_GRAIN_DEBUG_OFF ? 1 : 0, width, height, sc.s);
            }
        }
        if (e == cudaSuccess && debug != FJ_GRAIN_DEBUG_OFF)
            e = fjb::launch_grain_debug_average(density_c, density_m, density_y, ds, 0.5f, grain->debug_scale, width,
                                                height, sc.s);
        if (e != cudaSuccess) return cuda_status(e, error, "visual grain");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_visual_grain");
    }
}
