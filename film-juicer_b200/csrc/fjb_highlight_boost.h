// fjb_highlight_boost.h -- highlight reconstruction on the camera carrier planes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fjb {

// Dispositions in the reference's order (src/Cuda/Film/JuicerCudaHighlightBoost.h:17-22).
enum : int { kBoostBypass = 0, kBoostApplied = 1, kBoostInvalidCarrier = 2, kBoostPeakOverflow = 3 };

struct BoostDescriptor {
    double protection, sharpness, peak_gain;
};

// Device word block: frame maximum (float bits), invalid flag, disposition.
struct BoostState {
    unsigned maximum_bits;
    unsigned invalid;
    unsigned disposition;
    unsigned pad;
};

// Carrier planes B, G, R (`stride` floats per row) boosted in place; `state` is reset
// first and receives the disposition.
cudaError_t launch_highlight_boost(const BoostDescriptor& d, float* b, float* g, float* r, long long stride, int width,
                                   int height, BoostState* state, cudaStream_t stream);

} // namespace fjb
