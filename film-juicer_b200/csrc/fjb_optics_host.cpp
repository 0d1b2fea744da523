// fjb_optics_host.cpp -- FjScatterHalation -> the two fused optics passes.
//
// Descriptor validation restates native/juicer_cuda_descriptors.cpp:140-182 (FIR
// radius 1..9 with finite non-negative taps and zero padding; finite YVV
// coefficients; factored coefficients h in (0,1), t in (0,1), 0 < g < 2(1+t)).
// The per-channel schedule restates src/Cuda/Film/JuicerCudaScatterHalation.cu:
// 760-845: scatter is skipped when the scatter amount is zero, the tail Gaussians only
// run when the tail weight is positive, back-reflection is skipped when the channel's
// total strength is zero.
#include <cmath>
#include <cstring>

#include "fjb_optics.h"

namespace fjb {

namespace {

void segment_map(OpticGauss& g);

const float kTailAmplitudes[3] = {0.1633f, 0.6496f, 0.1870f};

bool decode_gauss(const FjHalationGaussian& s, OpticGauss& g) {
    std::memset(&g, 0, sizeof(g));
    const bool fir = s.kind == FJ_HALATION_FIR_REFLECT;
    if (s.kind > FJ_HALATION_YVV_REPLICATE_FACTORED) return false;
    if (fir ? (s.radius < 1 || s.radius > kOpticMaxFirRadius) : s.radius != 0) return false;
    const int taps = fir ? 2 * s.radius + 1 : 0;
    for (int i = 0; i < 19; ++i) {
        const float w = s.fir_weights[i];
        if (i < taps ? (!std::isfinite(w) || w < 0.0f) : (w != 0.0f || std::signbit(w))) return false;
    }
    if (s.kind == FJ_HALATION_YVV_REPLICATE || s.kind == FJ_HALATION_YVV_REPLICATE_FACTORED) {
        for (float v : s.yvv)
            if (!std::isfinite(v)) return false;
        if (s.kind == FJ_HALATION_YVV_REPLICATE_FACTORED &&
            (!(s.yvv[0] > 0.0f && s.yvv[0] < 1.0f && s.yvv[1] > 0.0f &&
               (double)s.yvv[1] < 2.0 * (1.0 + s.yvv[2]) && s.yvv[2] > 0.0f && s.yvv[2] < 1.0f) ||
             s.yvv[3] != 0.0f || std::signbit(s.yvv[3])))
            return false;
    } else {
        for (float v : s.yvv)
            if (v != 0.0f || std::signbit(v)) return false;
    }
    g.kind = (int)s.kind;
    g.radius = s.radius;
    std::memcpy(g.w, s.fir_weights, sizeof(g.w));
    std::memcpy(g.yvv, s.yvv, sizeof(g.yvv));
    segment_map(g);
    return true;
}

} // namespace

namespace {

int segments(int n) { return optic_segments(n); }

// The recursion's state map over kOpticSeg steps with zero input, in FP64: the
// operator that carries a segment's entry state to its exit state.
void segment_map(OpticGauss& g) {
    double m[9] = {0};
    if (g.kind == kGaussYvv) {
        // (s1, s2, s3) -> (B1 s1 + B2 s2 + B3 s3, s1, s2)
        const double m0[9] = {g.yvv[1], g.yvv[2], g.yvv[3], 1, 0, 0, 0, 1, 0};
        std::memcpy(m, m0, sizeof(m));
    } else if (g.kind == kGaussYvvFactored) {
        // s1' = (1-h) s1; s3' = t s3 + g (s1' - s2); s2' = s2 + s3'
        const double h = g.yvv[0], gg = g.yvv[1], t = g.yvv[2];
        const double m0[9] = {1 - h, 0, 0, gg * (1 - h), 1 - gg, t, gg * (1 - h), -gg, t};
        std::memcpy(m, m0, sizeof(m));
    } else {
        return;
    }
    double r[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int step = 1; step <= 4 * kOpticSeg; ++step) {
        double t[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) t[i * 3 + j] = m[i * 3] * r[j] + m[i * 3 + 1] * r[3 + j] + m[i * 3 + 2] * r[6 + j];
        std::memcpy(r, t, sizeof(r));
        if (step == kOpticSeg) std::memcpy(g.seg, r, sizeof(r));
    }
    std::memcpy(g.seg4, r, sizeof(r));
}

} // namespace

size_t halation_scratch_floats(int width, int height) {
    const size_t lines = (size_t)(width > height ? width : height);
    const size_t segs = (size_t)(segments(width) > segments(height) ? segments(width) : segments(height));
    return (size_t)3 * kOpticMaxGauss * (size_t)width * (size_t)height // row-filtered planes
           + (size_t)3 * kOpticMaxGauss * lines * segs * 3               // segment states
           + (size_t)2 * 3 * kOpticMaxGauss * lines;                     // edge values
}

bool scatter_halation(const FjScatterHalation& d, float* planes_rgb[3], long long stride, int width, int height,
                      float* scratch, cudaStream_t stream, std::string& why, cudaError_t& err) {
    err = cudaSuccess;
    if (d.bounce_count > FJ_HALATION_MAX_BOUNCES) {
        why = "scatter_halation.bounce_count exceeds 5";
        return false;
    }
    const size_t plane = (size_t)width * (size_t)height;
    OpticPass scatter{};
    OpticPass bounce{};
    scatter.width = bounce.width = width;
    scatter.height = bounce.height = height;
    {
        const int lines = width > height ? width : height;
        const int segs = segments(width) > segments(height) ? segments(width) : segments(height);
        float* tail = scratch + (size_t)3 * kOpticMaxGauss * plane;
        for (OpticPass* P : {&scatter, &bounce}) {
            P->lines_max = lines;
            P->segs_max = segs;
            P->carry = tail;
            P->edge_a = tail + (size_t)3 * kOpticMaxGauss * lines * segs * 3;
            P->edge_b = P->edge_a + (size_t)3 * kOpticMaxGauss * lines;
        }
    }
    for (int c = 0; c < 3; ++c) {
        const FjHalationChannel& ch = d.channels[c];
        float* temps[kOpticMaxGauss];
        for (int g = 0; g < kOpticMaxGauss; ++g) temps[g] = scratch + ((size_t)c * kOpticMaxGauss + g) * plane;
        if (d.scatter_amount != 0.0f) {
            OpticJob& J = scatter.job[scatter.jobs];
            std::memset(&J, 0, sizeof(J));
            J.src = planes_rgb[c];
            J.stride = stride;
            J.mode = kOpticScatter;
            J.tail_weight = ch.tail_weight;
            J.amount = d.scatter_amount;
            J.tail_count = ch.tail_weight > 0.0f ? 3 : 0;
            for (int i = 0; i < J.tail_count; ++i) {
                if (!decode_gauss(ch.tail[i], J.g[i])) {
                    why = "scatter_halation tail Gaussian is malformed";
                    return false;
                }
                J.coef[i] = kTailAmplitudes[i];
            }
            if (!decode_gauss(ch.core, J.g[J.tail_count])) {
                why = "scatter_halation core Gaussian is malformed";
                return false;
            }
            J.count = J.tail_count + 1;
            for (int g = 0; g < J.count; ++g) J.temp[g] = temps[g];
            ++scatter.jobs;
        }
        if (ch.total_strength != 0.0f && d.bounce_count > 0) {
            OpticJob& J = bounce.job[bounce.jobs];
            std::memset(&J, 0, sizeof(J));
            J.src = planes_rgb[c];
            J.stride = stride;
            J.mode = kOpticBounce;
            J.amount = ch.total_strength;
            J.renormalize = d.renormalize ? 1 : 0;
            J.count = (int)d.bounce_count;
            for (int b = 0; b < J.count; ++b) {
                if (!decode_gauss(ch.bounce[b], J.g[b])) {
                    why = "scatter_halation bounce Gaussian is malformed";
                    return false;
                }
                J.coef[b] = d.bounce_weights[b];
                J.temp[b] = temps[b];
            }
            ++bounce.jobs;
        } else if (ch.total_strength != 0.0f && d.renormalize) {
            // zero bounces with strength: plane / (1 + s) after adding nothing
            OpticJob& J = bounce.job[bounce.jobs];
            std::memset(&J, 0, sizeof(J));
            J.src = planes_rgb[c];
            J.stride = stride;
            J.mode = kOpticBounce;
            J.amount = ch.total_strength;
            J.renormalize = 1;
            J.count = 1;
            J.g[0].kind = kGaussIdentity;
            J.coef[0] = 0.0f;
            ++bounce.jobs;
        }
    }
    if (scatter.jobs) {
        err = launch_optic_pass(scatter, stream);
        if (err != cudaSuccess) {
            why = "scatter pass launch failed";
            return false;
        }
    }
    if (bounce.jobs) {
        err = launch_optic_pass(bounce, stream);
        if (err != cudaSuccess) {
            why = "back-reflection pass launch failed";
            return false;
        }
    }
    return true;
}

} // namespace fjb
