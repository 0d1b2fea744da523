// fjb_api_diffusion.cpp -- extern "C" entry point of the diffusion stage.
#include <cuda_runtime.h>

#include <cmath>

#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "fjb_diffusion.h"
#include "fjb_schedule.h"

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

namespace {

double ordered_max(double v, double floor_value) { return v > floor_value ? v : floor_value; }

struct Group {
    double lambda_um[4];
    double weights[4];
    int count;
};

// Log-spaced expansion of one PSF group (rust/film-juicer-core/src/optics/
// diffusion_frame.rs:285-334); bloom groups weight by lambda^(2 - alpha).
bool expand_group(double center, double spread, int count, bool bloom, double alpha, Group& g) {
    g = Group{};
    g.count = count;
    const double lo = std::log(center / spread), hi = std::log(center * spread);
    if (!std::isfinite(lo) || !std::isfinite(hi)) return false;
    for (int i = 0; i < count; ++i) {
        double l;
        if (i + 1 == count) {
            l = hi;
        } else if (i != 0) {
            const double t = (double)i / (double)(count - 1);
            l = lo + (hi - lo) * t;
        } else {
            l = lo;
        }
        g.lambda_um[i] = std::exp(l);
        g.weights[i] = bloom ? std::pow(g.lambda_um[i], 2.0 - alpha) : 1.0;
        if (!(std::isfinite(g.lambda_um[i]) && g.lambda_um[i] > 0.0 && std::isfinite(g.weights[i]) &&
              g.weights[i] >= 0.0))
            return false;
    }
    double total = 0.0;
    for (int i = 0; i < count; ++i) total += g.weights[i];
    if (!(std::isfinite(total) && total > 0.0)) return false;
    for (int i = 0; i < count; ++i) g.weights[i] /= total;
    return true;
}

} // namespace

// Nine PSF components of a diffusion filter sample (restates
// rust/film-juicer-core/src/optics/diffusion_frame.rs:238-421, the host preparation the
// reference reaches through fj_diffusion_components_prepare): core (2 components,
// spread 1.5), halo (3, spread 2, per-channel warmth tilt on axes 1.30 / 0.15 / -1.45),
// bloom (4, spread 2.5, weights lambda^(2 - alpha), alpha by family).
extern "C" FjStatus fjb_diffusion_components_host(const FjDiffusion* d, FjDiffusionComponents* out,
                                                  FjErrorBuffer* error) {
    if (!d || !out) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    if (d->family > FJ_DIFFUSION_CINEBLOOM) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "family");
    double total = 0.0;
    for (double w : d->group_weights) {
        if (!std::isfinite(w) || w < 0.0) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "group weights");
        total += w;
    }
    if (!(std::isfinite(total) && total > 0.0))
        return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "group weights");
    for (double c : d->group_lambda_um)
        if (!(std::isfinite(c) && c > 0.0)) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "group centers");
    if (!std::isfinite(d->warmth) || d->warmth < -1.5 || d->warmth > 1.5)
        return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "warmth");
    if (!(std::isfinite(d->spatial_scale) && d->spatial_scale > 0.0) ||
        !(std::isfinite(d->pixel_size_um) && d->pixel_size_um > 0.0) || d->radius_px <= 0)
        return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "scale, pixel size or radius");
    const double alphas[4] = {3.2, 3.5, 2.9, 2.5};
    Group core, halo, bloom;
    if (!expand_group(d->group_lambda_um[0], 1.5, 2, false, 0.0, core) ||
        !expand_group(d->group_lambda_um[1], 2.0, 3, false, 0.0, halo) ||
        !expand_group(d->group_lambda_um[2], 2.5, 4, true, alphas[d->family], bloom))
        return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "component expansion");
    // halo channel tilt
    double grad[4] = {0, 0, 0, 0}, target = 0.0, wgrad = 0.0;
    for (int i = 0; i < halo.count; ++i) {
        grad[i] = -1.0 + 2.0 * (double)i / (double)(halo.count - 1);
        target += halo.weights[i];
        wgrad += halo.weights[i] * grad[i];
    }
    if (!(std::isfinite(target) && target > 0.0))
        return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "halo channel weights");
    wgrad /= target;
    for (int i = 0; i < halo.count; ++i) grad[i] -= wgrad;
    double halo_rgb[3][4] = {};
    const double axes[3] = {1.30, 0.15, -1.45};
    for (int c = 0; c < 3; ++c) {
        double t = 0.0;
        for (int i = 0; i < halo.count; ++i) {
            halo_rgb[c][i] = ordered_max(halo.weights[i] * (1.0 + d->warmth * axes[c] * grad[i]), 0.0);
            t += halo_rgb[c][i];
        }
        if (t > 0.0) {
            const double s = target / t;
            for (int i = 0; i < halo.count; ++i) halo_rgb[c][i] *= s;
        } else {
            for (int i = 0; i < halo.count; ++i) halo_rgb[c][i] = halo.weights[i];
        }
    }
    const double scale = ordered_max(d->spatial_scale, 1e-6);
    const Group* groups[3] = {&core, &halo, &bloom};
    int off = 0;
    for (int gi = 0; gi < 3; ++gi) {
        const Group& g = *groups[gi];
        for (int i = 0; i < g.count; ++i) {
            const int o = off + i;
            out->lambda_px[o] = ordered_max(g.lambda_um[i] * scale / d->pixel_size_um, 1e-6);
            if (gi == 1) {
                out->red_weights[o] = d->group_weights[1] * halo_rgb[0][i];
                out->green_weights[o] = d->group_weights[1] * halo_rgb[1][i];
                out->blue_weights[o] = d->group_weights[1] * halo_rgb[2][i];
            } else {
                const double w = d->group_weights[gi] * g.weights[i];
                out->red_weights[o] = out->green_weights[o] = out->blue_weights[o] = w;
            }
        }
        off += g.count;
    }
    for (int o = 0; o < 9; ++o) {
        const double w[3] = {out->red_weights[o], out->green_weights[o], out->blue_weights[o]};
        bool bad = !(std::isfinite(out->lambda_px[o]) && out->lambda_px[o] > 0.0);
        for (double v : w) bad = bad || !std::isfinite(v) || v < 0.0;
        if (bad) return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "component output");
    }
    write_error(error, "");
    return ok_status();
}

extern "C" FjStatus fjb_diffusion(const FjDiffusionComponents* components, int32_t radius_px, double scatter_fraction,
                                  const float* src_r, const float* src_g, const float* src_b, float* dst_r,
                                  float* dst_g, float* dst_b, ptrdiff_t stride, int32_t width, int32_t height,
                                  void* stream, FjErrorBuffer* error) {
    try {
        if (!components || !src_r || !src_g || !src_b || !dst_r || !dst_g || !dst_b)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (width <= 0 || height <= 0) {
            write_error(error, "");
            return ok_status();
        }
        if (stride < width) return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "stride below width");
        if (dst_r == src_r || dst_g == src_g || dst_b == src_b)
            return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "diffusion output must not alias its input");
        if (!(scatter_fraction >= 0.0 && scatter_fraction <= 1.0))
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "diffusion scatter fraction outside [0, 1]");
        for (int k = 0; k < 9; ++k)
            if (!(components->lambda_px[k] > 0.0) || !std::isfinite(components->lambda_px[k]))
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "diffusion lambda must be positive");
        const double* weights[3] = {components->red_weights, components->green_weights, components->blue_weights};
        std::vector<float> rows[3];
        int taps = 0;
        std::string why;
        for (int c = 0; c < 3; ++c)
            if (!fjb::diffusion_psf_rows(components->lambda_px, weights[c], radius_px, rows[c], taps, why))
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        float* d_psf = nullptr;
        const size_t n = rows[0].size();
        cudaError_t e = cudaMalloc(&d_psf, 3 * n * sizeof(float));
        for (int c = 0; c < 3 && e == cudaSuccess; ++c)
            e = cudaMemcpyAsync(d_psf + c * n, rows[c].data(), n * sizeof(float), cudaMemcpyHostToDevice, s);
        float* d_fft = nullptr; // FFT form: PSF spectrum, then the row-spectrum workspace
        if (e == cudaSuccess) {
            const float* psf[3] = {d_psf, d_psf + n, d_psf + 2 * n};
            float* dst[3] = {dst_r, dst_g, dst_b};
            const float* src[3] = {src_r, src_g, src_b};
            fjb::DiffusionFftPlan plan;
            if (fjb::diffusion_prefers_fft(width, height, radius_px) &&
                fjb::diffusion_fft_plan(width, height, radius_px, plan)) {
                e = cudaMalloc(&d_fft, (plan.spectrum_floats + plan.work_floats) * sizeof(float));
                float* work = d_fft + plan.spectrum_floats;
                if (e == cudaSuccess) e = fjb::launch_diffusion_fft_spectrum(plan, psf, taps, d_fft, work, s);
                if (e == cudaSuccess)
                    e = fjb::launch_diffusion_fft(plan, d_fft, (float)scatter_fraction, dst, src, stride, work, s);
            } else {
                e = fjb::launch_diffusion(psf, radius_px, taps, (float)scatter_fraction, dst, src, stride, width,
                                          height, s);
            }
        }
        // the host rows and the device buffers must outlive the copies and the kernels
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (d_psf) cudaFree(d_psf);
        if (d_fft) cudaFree(d_fft);
        if (e != cudaSuccess) return cuda_status(e, error, "diffusion");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_diffusion");
    }
}
