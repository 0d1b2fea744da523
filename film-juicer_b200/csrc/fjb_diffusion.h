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

// FFT form (fjb_diffusion_fft.cu), used from kDiffusionFftMinRadius up: the
// reflect-extended frame convolved circularly on an nx x ny power-of-two grid.
constexpr int kDiffusionFftMinRadius = 8;

struct DiffusionFftPlan {
    int width, height, radius;
    int m, log2m;     // nx / 2 complex points per row transform
    int ny, log2ny;   // column transform length 2^a 3^ny3 (log2ny: a when ny3 == 0, else -1)
    int ny3;          // factors of 3 in ny (0, 1 or 2)
    int ntw, log2ntw; // row twiddle table length (nx)
    int ey;           // extended rows H + 2r
    int sy;           // rows per spectrum column in the work buffer (ey rounded up to 4)
    int rows_per_cta, cols_per_cta; // powers of two
    int log2_rows_per_cta;
    size_t work_floats;     // 3 channels x (m + 1) x sy complex
    size_t spectrum_floats; // twiddles (2 ntw + 2 ny) + 3 channels x (m + 1) x ny reals
};

// False when the frame is too large for the transforms (then the direct form runs).
bool diffusion_fft_plan(int width, int height, int radius, DiffusionFftPlan& plan);
bool diffusion_prefers_fft(int width, int height, int radius);

// PSF spectrum (and twiddle table) of the PSF rows into `spectrum`
// (plan.spectrum_floats floats); `work` holds plan.work_floats floats.
cudaError_t launch_diffusion_fft_spectrum(const DiffusionFftPlan& plan, const float* const psf_rows[3], int taps,
                                          float* spectrum, float* work, cudaStream_t stream);

// dst[c] = (1 - fraction) src[c] + fraction (PSF_c * src[c]) through the spectrum.
cudaError_t launch_diffusion_fft(const DiffusionFftPlan& plan, const float* spectrum, float fraction, float* dst[3],
                                 const float* src[3], long long stride, float* work, cudaStream_t stream);

} // namespace fjb
