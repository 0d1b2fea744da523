// fjb_optics.h -- parameter blocks of the separable optics passes (scatter/halation).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <string>

#include "../../include/juicer_cuda_api.h"

namespace fjb {

// Gaussian operator kinds, numbered as FJ_HALATION_* in the C-ABI.
enum GaussKind : int { kGaussIdentity = 0, kGaussFir = 1, kGaussYvv = 2, kGaussYvvFactored = 3 };

constexpr int kOpticMaxGauss = 5;
constexpr int kOpticMaxFirRadius = 9;

constexpr int kOpticSeg = 64; // segment length of the block-parallel recursions

struct OpticGauss {
    int kind;
    int radius;   // FIR only
    float w[19];  // FIR weights, w[radius] is the centre tap
    float yvv[4]; // legacy: B, B1, B2, B3; factored: h, g, t, 0
    double seg[9]; // recursive kinds: the state map over kOpticSeg zero-input steps (row-major 3x3)
    double seg4[9]; // the same over 4 kOpticSeg steps
};

enum OpticMode : int { kOpticScatter = 0, kOpticBounce = 1 };

// One channel plane and the Gaussians evaluated on it in one sweep.
struct OpticJob {
    float* src;        // carrier plane, read, then overwritten by the combination
    long long stride;  // floats per row of src
    float* temp[kOpticMaxGauss]; // row-filtered planes, width floats per row
    int count;         // Gaussians in g[]
    OpticGauss g[kOpticMaxGauss];
    float coef[kOpticMaxGauss]; // tail amplitudes (scatter) or bounce weights (bounce)
    int mode;          // OpticMode
    int tail_count;    // scatter: g[0..tail_count) are tails, g[tail_count] is the core
    float tail_weight; // scatter only
    float amount;      // scatter amount, or bounce total strength
    int renormalize;   // bounce only
};

struct OpticPass {
    int width, height, jobs;
    OpticJob job[3];
    // block-parallel recursion buffers: 3 floats of segment state per (job, Gaussian,
    // line, segment) and two per-line edge values per (job, Gaussian, line)
    float* carry;
    float* edge_a;
    float* edge_b;
    int lines_max, segs_max;
};

cudaError_t launch_optic_pass(const OpticPass& P, cudaStream_t stream);

// Segments of the block-parallel recursions along a line of n samples.
int optic_segments(int n);

// Scratch floats needed by scatter_halation for a width x height frame.
size_t halation_scratch_floats(int width, int height);

// Runs scatter then back-reflection on the three carrier planes (R, G, B order of the
// descriptor's channels). `scratch` holds halation_scratch_floats() floats.
bool scatter_halation(const FjScatterHalation& d, float* planes_rgb[3], long long stride, int width, int height,
                      float* scratch, cudaStream_t stream, std::string& why, cudaError_t& err);

} // namespace fjb
