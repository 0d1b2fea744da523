// fjb_dir.h -- spatial DIR (development-inhibitor-releasing coupler) diffusion (a7).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/juicer_cuda_api.h"

namespace fjb {

enum DirOperator : int { kDirOpNone = 0, kDirOpIdentity = 1, kDirOpFir = 2, kDirOpYvv = 3 };
constexpr int kDirMaxComponents = 4;
constexpr int kDirMaxFirRadius = 64;

// Reflected-boundary start weights and end matrix of one axis of a recursive
// Gaussian (restatement of rust/film-juicer-core/src/film/dir/boundary.rs:362-490).
struct DirAxisBoundary {
    std::vector<double> weights; // 3 rows x length, row-major (state history 0, 1, 2)
    int length = 0;
    int terminal_size = 0;
    double terminal[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
};

// Returns false with `why` when the boundary system is singular or the weights fail
// the record's certification tolerance.
bool dir_axis_boundary(const FjDirGaussian& g, int axis_length, DirAxisBoundary& out, std::string& why);

// Normalized Gaussian taps for radius r (restatement of
// rust/film-juicer-core/src/optics/gaussian.rs:16-52): f64 exponentials narrowed to f32,
// then scaled by the f64 reciprocal of their f64 sum.
std::vector<float> gaussian_taps(int radius, float sigma_px);

struct DirComponentDev {
    int op;
    float weight;
    int radius;
    const float* taps; // device, 2r+1
    int symmetric_taps; // taps[i] == taps[2r - i] bit for bit
    double ff;
    double fb[3];
    const double* h_init;
    int h_len, h_tsize;
    double h_term[9];
    const double* v_init;
    int v_len, v_tsize;
    double v_term[9];
    double seg[9]; // recursion state map over kDirSeg zero-input steps (row-major 3x3)
    double seg4[9]; // the same over 4 kDirSeg steps
    // Factored FP32 form of the recursion (factored != 0): a unit-DC first-order section
    // u += c0 (x - u) into the second-order section v = c2 v + c1 (u - y), y += v, with
    // state (u, y, v); to_fac / from_fac map direct states (y[n-1], y[n-2], y[n-3]) to it
    // and back, seg_f / seg4_f are its zero-input maps over kDirSeg and 4 kDirSeg steps.
    int factored;
    float fac[3];
    double to_fac[9], from_fac[9];
    double seg_f[9], seg4_f[9];
};

constexpr int kDirSeg = 64; // segment length of the block-parallel recursions

struct DirBlurParams {
    int width, height, count;
    DirComponentDev comp[kDirMaxComponents];
    const float* raw[3]; // correction planes Y, M, C (width floats per row)
    float* filtered[3];  // outputs Y, M, C
    float* temp[3][kDirMaxComponents];
    // block-parallel recursion buffers: 3 doubles of segment state per (channel,
    // component, line, segment); 9 doubles of start states and end block per
    // (channel, component, line)
    double* carry;
    double* start;
    int lines_max, segs_max;
};

// Bytes of the recursion buffers for a width x height frame.
size_t dir_recursion_bytes(int width, int height);

// Segments of the block-parallel recursions along a line of n samples.
int dir_segments(int n);

cudaError_t launch_dir_blur(const DirBlurParams& p, cudaStream_t stream);

// Device-resident operator tables for one frame geometry.
struct DirPlan {
    int width = 0, height = 0, count = 0;
    DirComponentDev comp[kDirMaxComponents] = {};
    std::vector<void*> owned;
    void release();
};

bool dir_plan_create(const FjSpatialDir& sd, int width, int height, cudaStream_t stream, DirPlan& plan,
                     std::string& why, cudaError_t& err);

size_t dir_scratch_floats(int width, int height);

} // namespace fjb

struct FjbRecipe;

namespace fjb {

// Spatial-DIR source + blur with a prepared plan (enqueues only; the plan must stay
// alive until the work has run).
FjStatus spatial_dir_apply(FjbRecipe* recipe, const DirPlan& plan, const float* src, ptrdiff_t src_row_bytes,
                           uint32_t components, const float* carrier_b, const float* carrier_g, const float* carrier_r,
                           ptrdiff_t carrier_stride, int width, int height, float* filtered_y, float* filtered_m,
                           float* filtered_c, float* log_raw_b, float* log_raw_g, float* log_raw_r, float* scratch,
                           size_t scratch_bytes, void* stream, FjErrorBuffer* error);

} // namespace fjb
