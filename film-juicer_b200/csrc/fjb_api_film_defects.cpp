// fjb_api_film_defects.cpp -- film and gate defects: record validation and the
// extern "C" stage entries.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "fjb_film_defects.h"
#include "fjb_internal.h"
#include "fjb_scanner_post.h"
#include "fjb_schedule.h"

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

namespace fjb {

namespace {

constexpr uint32_t kEffectsFlags =
    FJ_EFFECTS_WEAVE | FJ_EFFECTS_FILM | FJ_EFFECTS_GATE_TRANSMITTANCE | FJ_EFFECTS_GATE_OUTPUT | FJ_EFFECTS_FULL_FRAME;

// Candidates a 32 x 8 tile visits in one family is bounded before launch: the cell
// range of a tile grows with the support and shrinks with the cell size, and a record
// whose range would be enormous (or not finite) is rejected instead of run.
constexpr double kMaxCandidatesPerTile = 1 << 16;

bool family_ok(float probability, float cw, float ch, float support_x, float support_y, float softness_max,
               float step_x, float step_y, const char* name, std::string& why) {
    if (!(probability > 0.0f)) return true;
    const bool finite = std::isfinite(cw) && std::isfinite(ch) && std::isfinite(support_x) &&
                        std::isfinite(support_y) && std::isfinite(softness_max) && std::isfinite(step_x) &&
                        std::isfinite(step_y);
    if (!finite || !(cw > 0.0f) || !(ch > 0.0f) || !(step_x > 0.0f) || !(step_y > 0.0f)) {
        why = std::string("film effects: ") + name + " cell size or sample step not positive and finite";
        return false;
    }
    const double sx = std::fabs((double)support_x + softness_max), sy = std::fabs((double)support_y + softness_max);
    const double columns = (32.0 * step_x + 2.0 * sx) / cw + 3.0;
    const double rows = (8.0 * step_y + 2.0 * sy) / ch + 3.0;
    if (!(columns * rows * 2.0 <= kMaxCandidatesPerTile)) {
        why = std::string("film effects: ") + name + " cells too small for the support (too many candidates per tile)";
        return false;
    }
    return true;
}

} // namespace

bool effects_plan_from(const FjFilmEffects& e, EffectsPlan& plan, std::string& why) {
    plan = EffectsPlan{};
    if ((e.flags & ~kEffectsFlags) != 0) {
        why = "film effects: unknown flags";
        return false;
    }
    if ((e.flags & (FJ_EFFECTS_FILM | FJ_EFFECTS_GATE_OUTPUT)) == 0) {
        if (e.flags == 0 && e.hash == 0 && e.recipe_hash == 0) return true;
        why = "film effects: inactive record carries flags or an identity";
        return false;
    }
    if (e.hash == 0 || e.recipe_hash == 0) {
        why = "film effects: active record without its identity hashes";
        return false;
    }
    plan.film = (e.flags & FJ_EFFECTS_FILM) != 0;
    plan.gate_output = (e.flags & FJ_EFFECTS_GATE_OUTPUT) != 0;
    plan.weave = plan.gate_output && (e.flags & FJ_EFFECTS_WEAVE) != 0;
    plan.gate_mask = plan.gate_output && (e.flags & FJ_EFFECTS_GATE_TRANSMITTANCE) != 0;
    plan.full_frame = (e.flags & FJ_EFFECTS_FULL_FRAME) != 0;
    plan.film_dust = plan.film && e.film_dust.slot_probability > 0.0f;
    const float sx = e.sample_step_x_mm, sy = e.sample_step_y_mm;
    for (const FjDefectOrigin& o : e.origins)
        if (!std::isfinite(o.local_x_mm) || !std::isfinite(o.local_y_mm)) {
            why = "film effects: defect origin not finite";
            return false;
        }
    if (plan.film) {
        if (!family_ok(e.film_dust.slot_probability, e.film_dust.cell_width_mm, e.film_dust.cell_height_mm,
                       e.film_dust.support_x_mm, e.film_dust.support_y_mm, e.film_dust.softness_max_mm, sx, sy,
                       "film dust", why) ||
            !family_ok(e.film_scratch.slot_probability, e.film_scratch.cell_width_mm, e.film_scratch.cell_height_mm,
                       e.film_scratch.support_x_mm, e.film_scratch.support_y_mm, e.film_scratch.softness_max_mm, sx,
                       sy, "film scratch", why))
            return false;
    }
    if (plan.gate_mask) {
        if (e.gate_width <= 0 || e.gate_height <= 0) {
            why = "film effects: gate transmittance without a gate grid";
            return false;
        }
        if (!family_ok(e.gate_dust.slot_probability, e.gate_dust.cell_width_mm, e.gate_dust.cell_height_mm,
                       e.gate_dust.support_x_mm, e.gate_dust.support_y_mm, e.gate_dust.softness_max_mm, 2.0f * sx,
                       2.0f * sy, "gate dust", why) ||
            !family_ok(e.gate_scratch.slot_probability, e.gate_scratch.cell_width_mm, e.gate_scratch.cell_height_mm,
                       e.gate_scratch.support_x_mm, e.gate_scratch.support_y_mm, e.gate_scratch.softness_max_mm,
                       2.0f * sx, 2.0f * sy, "gate scratch", why))
            return false;
    }
    return true;
}

} // namespace fjb

extern "C" {

size_t fjb_film_defects_scratch_bytes(const FjFilmEffects* effects, int32_t width, int32_t height) {
    return effects ? fjb::film_defects_table_bytes(*effects, width, height) : 0;
}

size_t fjb_gate_mask_scratch_bytes(const FjFilmEffects* effects, int32_t gate_width, int32_t gate_height) {
    return effects ? fjb::gate_mask_table_bytes(*effects, gate_width, gate_height) : 0;
}

FjStatus fjb_film_defects(const FjFilmEffects* effects, int32_t width, int32_t height, float* density_c,
                          float* density_m, float* density_y, float* dust, void* scratch, size_t scratch_bytes,
                          void* stream, FjErrorBuffer* error) {
    try {
        if (!effects || !density_c || !density_m || !density_y)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        fjb::EffectsPlan plan;
        std::string why;
        if (!fjb::effects_plan_from(*effects, plan, why)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        if (!plan.film) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "film effects: film defects are off");
        if (plan.film_dust && !dust)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "film dust needs a transmittance plane");
        if (width < 0 || height < 0) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "negative frame size");
        cudaError_t e = fjb::launch_film_defects(*effects, width, height, density_c, density_m, density_y,
                                                 plan.film_dust ? dust : nullptr, reinterpret_cast<cudaStream_t>(stream),
                                                 scratch, scratch_bytes);
        if (e != cudaSuccess) return cuda_status(e, error, "film defects");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_film_defects");
    }
}

FjStatus fjb_gate_mask(const FjFilmEffects* effects, float* gate_mask, int32_t gate_width, int32_t gate_height,
                       void* scratch, size_t scratch_bytes, void* stream, FjErrorBuffer* error) {
    try {
        if (!effects || !gate_mask) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        fjb::EffectsPlan plan;
        std::string why;
        if (!fjb::effects_plan_from(*effects, plan, why)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        if (!plan.gate_mask)
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "film effects: gate transmittance is off");
        if (gate_width <= 0 || gate_height <= 0)
            return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "gate grid must be non-empty");
        cudaError_t e = fjb::launch_gate_mask(*effects, gate_mask, gate_width, gate_height,
                                              reinterpret_cast<cudaStream_t>(stream), scratch, scratch_bytes);
        if (e != cudaSuccess) return cuda_status(e, error, "gate mask");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_gate_mask");
    }
}

FjStatus fjb_render_from_density_effects(FjbRecipe* recipe, const FjScannerPostEffects* post, uint64_t glare_seed,
                                         int32_t glare_origin_x, int32_t glare_origin_y,
                                         const FjFilmEffects* effects, const float* dust, const float* gate_mask,
                                         const float* density_c, const float* density_m, const float* density_y,
                                         const float* src, ptrdiff_t src_row_bytes, float* dst,
                                         ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                         float* scratch, size_t scratch_bytes, void* stream, FjErrorBuffer* error) {
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
        fjb::OutputEffects fx;
        if (effects) {
            fjb::EffectsPlan ep;
            if (!fjb::effects_plan_from(*effects, ep, why)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
            if (ep.film_dust && !dust)
                return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "film dust needs its transmittance plane");
            if (ep.gate_mask && !gate_mask)
                return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "gate transmittance needs the gate mask");
            fx.dust = ep.film_dust ? dust : nullptr;
            fx.weave = ep.weave;
            fx.weave_dx = effects->weave_dx_px;
            fx.weave_dy = effects->weave_dy_px;
            fx.weave_cos = effects->weave_cos_rot;
            fx.weave_sin = effects->weave_sin_rot;
            fx.gate_mask = ep.gate_mask ? gate_mask : nullptr;
            fx.gate_w = ep.gate_mask ? effects->gate_width : 0;
            fx.gate_h = ep.gate_mask ? effects->gate_height : 0;
            fx.roi_x = effects->roi_offset_x;
            fx.roi_y = effects->roi_offset_y;
        }
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
                                             height, components, scratch, taps, s, error, fx);
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_render_from_density_effects");
    }
}

} // extern "C"
