// fjb_diffusion.h -- camera / enlarger diffusion (direct radially symmetric PSF).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace fjb {

constexpr int kMaxDiffusionRadius = 80; // shared-memory tile limit of the direct kernel

// Normalised PSF rows |dy| = 0..radius, each (2r+1) taps padded with zeros to `taps`
// (a multiple of 16).
bool diffusion_psf_rows(const double lambda_px[9], const double weights[9], int radius, std::vector<float>& rows,
                        int& taps, std::string& why);

size_t diffusion_smem_bytes(int radius);

// dst[c] = (1 - fraction) src[c] + fraction (PSF_c * src[c]); dst must not alias src.
cudaError_t launch_diffusion(const float* const psf_rows[3], int radius, int taps, float fraction, float* dst[3],
                             const float* src[3], long long stride, int width, int height, cudaStream_t stream);

} // namespace fjb
