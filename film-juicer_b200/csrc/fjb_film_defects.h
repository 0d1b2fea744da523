// fjb_film_defects.h -- procedural film and gate defects (dust, scratches).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/juicer_cuda_api.h"

namespace fjb {

// Film dust and film scratches at the frame's pixels (full-frame pixel = pixel + ROI
// offset): the dust transmittance plane (required when film dust is on) and, when film
// scratches are on, the C, M, Y density planes scaled by the retained fraction.
// `table` (table_bytes, may be null): device memory for the frame's particle table,
// film_defects_table_bytes(e, width, height) bytes; without it the tiles build their
// candidates themselves (same results, slower).
cudaError_t launch_film_defects(const FjFilmEffects& e, int width, int height, float* c, float* m, float* y,
                                float* dust_out, cudaStream_t stream, void* table = nullptr, size_t table_bytes = 0);
size_t film_defects_table_bytes(const FjFilmEffects& e, int width, int height);

// Gate dust x gate scratch transmittance at the gate grid (width x height, twice the
// sample step).
cudaError_t launch_gate_mask(const FjFilmEffects& e, float* mask, int width, int height, cudaStream_t stream,
                             void* table = nullptr, size_t table_bytes = 0);
size_t gate_mask_table_bytes(const FjFilmEffects& e, int width, int height);

// The effects record's stage switches, after validation.
struct EffectsPlan {
    bool film = false;         // film dust / scratches on the capture density
    bool film_dust = false;    // the dust transmittance plane is needed
    bool gate_output = false;  // weave and / or the gate mask at the output encoding
    bool weave = false;
    bool gate_mask = false;
    bool full_frame = false;
};

// Validates an effects record as the reference's descriptor decoding does
// (native/juicer_cuda_descriptors.cpp:467-515): known flags; an inactive record is all
// zero; an active one carries its identity hashes.
bool effects_plan_from(const FjFilmEffects& e, EffectsPlan& plan, std::string& why);

} // namespace fjb
