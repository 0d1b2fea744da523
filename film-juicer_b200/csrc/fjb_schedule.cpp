// fjb_schedule.cpp -- fj_cuda_* lifecycle and the per-frame stage schedule.
//
// Lifecycle and admission rules restate native/juicer_cuda_api.cpp:245-600:
// create publishes exactly one owner, a second live owner is rejected; shutdown
// releases device state and leaves a closed handle; destroy consumes the handle.
// The render schedule restates the stage order of
// src/Cuda/JuicerCudaExecutor.cpp:2561 (direct) and :2831 (print); frames without a
// spatial stage run as one fused launch (the reference's Monolithic capture,
// src/Cuda/Scan/JuicerCudaScanPipeline.cu:3771).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "../../include/juicer_cuda_api.h"
#include "fjb_diffusion.h"
#include "fjb_highlight_boost.h"
#include "fjb_film_defects.h"
#include "fjb_scanner_post.h"
#include "fjb_dir.h"
#include "fjb_internal.h"
#include "fjb_recipe.h"
#include "fjb_schedule.h"

namespace fjb_sched {
// Device tables of one diffusion stage for one descriptor and frame size: the PSF rows
// and, for the FFT form, the PSF spectrum.
struct DiffusionCache {
    float* psf = nullptr;
    size_t psf_bytes = 0;
    uint64_t key = 0;
    int taps = 0;
    float* spectrum = nullptr;
    size_t spectrum_bytes = 0;
    uint64_t spectrum_key = 0;
    void release() {
        if (psf) cudaFree(psf);
        if (spectrum) cudaFree(spectrum);
        *this = DiffusionCache{};
    }
};

// A device copy of host floats (the scanner post effects' Gaussian taps).
struct DeviceFloats {
    float* data = nullptr;
    size_t bytes = 0;
    void release() {
        if (data) cudaFree(data);
        *this = DeviceFloats{};
    }
};

// Owner caches hold at most this many entries each; a full cache is emptied (after
// the device has drained) before a new entry is added.
constexpr size_t kCacheEntries = 32;
} // namespace fjb_sched

struct FjCuda {
    std::mutex gate;
    bool closed = false;
    int device = -1;
    std::map<uint64_t, FjbRecipe*> recipes; // keyed by recipe_hash (non-zero only)
    void* work = nullptr;                    // frame workspace: planes + stage scratch
    size_t work_bytes = 0;
    float* ae_scale = nullptr;               // device auto-exposure scale
    FjbNoise* noise = nullptr;               // device copy of the static grain noise
    uintptr_t noise_key[3] = {0, 0, 0};
    std::map<uint64_t, fjb::DirPlan> dir_plans;                 // spatial-DIR operator tables per geometry
    std::map<uint64_t, fjb_sched::DiffusionCache> diffusion;    // per (stage, descriptor, frame size)
    float* diffusion_fft_work = nullptr;     // FFT form: transposed row spectra of the frame (both stages)
    size_t diffusion_fft_work_bytes = 0;
    void* boost_state = nullptr;             // highlight reconstruction: frame maximum and disposition
    std::map<uint64_t, fjb_sched::DeviceFloats> post_taps;      // scanner post-effect taps per descriptor hash
    int32_t print_form = 0;                  // FJB_PRINT_* applied to every recipe rendered
    // diffusion form per (frame size, radius): measured once when autotuning is on
    bool autotune = false;
    std::map<uint64_t, int32_t> diffusion_form;
    // batches: per-frame flag words (device and pinned host), highlight states, the
    // instantiated graph of the last captured batch and its caller token
    uint32_t* batch_flags = nullptr;
    uint32_t* batch_flags_host = nullptr;
    size_t batch_slots = 0;
    std::vector<void*> batch_boost;
    cudaGraphExec_t batch_exec = nullptr;
    uint64_t batch_token = 0;
    int32_t batch_frames = 0;
    bool capturing = false;
    // optional per-stage device timing (CUDA events on the render stream)
    bool timing = false;
    bool timing_events = false;
    cudaEvent_t stage_ev[2 * FJB_STAGE_COUNT] = {};
    bool stage_open[FJB_STAGE_COUNT] = {};
    double stage_ms[FJB_STAGE_COUNT] = {};
    uint64_t stage_frames[FJB_STAGE_COUNT] = {};
};

namespace {

std::atomic<FjCuda*> g_live_owner{nullptr};

bool image_ok(const FjImage& im) {
    return im.address != 0 && (im.components == FJ_COMPONENTS_RGB || im.components == FJ_COMPONENTS_RGBA) &&
           im.depth == FJ_DEPTH_FLOAT32 && im.bounds.x2 >= im.bounds.x1 && im.bounds.y2 >= im.bounds.y1 &&
           im.row_bytes >= (ptrdiff_t)(im.bounds.x2 - im.bounds.x1) * (ptrdiff_t)im.components * 4;
}

bool rect_inside(const FjRect& inner, const FjRect& outer) {
    return inner.x1 >= outer.x1 && inner.y1 >= outer.y1 && inner.x2 <= outer.x2 && inner.y2 <= outer.y2;
}

const char* pixel_address(const FjImage& im, int x, int y) {
    return reinterpret_cast<const char*>(im.address) + (ptrdiff_t)(y - im.bounds.y1) * im.row_bytes +
           (ptrdiff_t)(x - im.bounds.x1) * (ptrdiff_t)im.components * 4;
}

bool aborted(const FjAbortCallback& cb) { return cb.query && cb.query(cb.user) == FJ_ABORT_REQUESTED; }

void stage_events_release(FjCuda* cuda);
void batch_graph_release(FjCuda* cuda);

void release_all(FjCuda* cuda) {
    for (auto& kv : cuda->recipes) {
        kv.second->r.release();
        delete kv.second;
    }
    cuda->recipes.clear();
    if (cuda->work) cudaFree(cuda->work);
    cuda->work = nullptr;
    cuda->work_bytes = 0;
    if (cuda->ae_scale) cudaFree(cuda->ae_scale);
    cuda->ae_scale = nullptr;
    if (cuda->noise) fjb_noise_destroy(cuda->noise, nullptr);
    cuda->noise = nullptr;
    batch_graph_release(cuda);
    for (auto& kv : cuda->dir_plans) kv.second.release();
    cuda->dir_plans.clear();
    for (auto& kv : cuda->diffusion) kv.second.release();
    cuda->diffusion.clear();
    if (cuda->diffusion_fft_work) cudaFree(cuda->diffusion_fft_work);
    cuda->diffusion_fft_work = nullptr;
    cuda->diffusion_fft_work_bytes = 0;
    if (cuda->boost_state) cudaFree(cuda->boost_state);
    cuda->boost_state = nullptr;
    for (auto& kv : cuda->post_taps) kv.second.release();
    cuda->post_taps.clear();
    cuda->diffusion_form.clear();
    if (cuda->batch_flags) cudaFree(cuda->batch_flags);
    if (cuda->batch_flags_host) cudaFreeHost(cuda->batch_flags_host);
    cuda->batch_flags = nullptr;
    cuda->batch_flags_host = nullptr;
    cuda->batch_slots = 0;
    for (void* b : cuda->batch_boost) cudaFree(b);
    cuda->batch_boost.clear();
    stage_events_release(cuda);
}

// The instantiated batch graph references owner buffers: it is dropped whenever one of
// them is freed or regrown.
void batch_graph_release(FjCuda* cuda) {
    if (cuda->batch_exec) cudaGraphExecDestroy(cuda->batch_exec);
    cuda->batch_exec = nullptr;
    cuda->batch_token = 0;
    cuda->batch_frames = 0;
}

// Makes room for one more entry in an owner cache (emptying a full one after the
// device has drained, which also invalidates a captured batch graph).
template <typename Map>
void cache_room(FjCuda* cuda, Map& m) {
    if (m.size() < fjb_sched::kCacheEntries) return;
    cudaDeviceSynchronize();
    batch_graph_release(cuda);
    for (auto& kv : m) kv.second.release();
    m.clear();
}

// Grows an owner buffer to at least `bytes` (contents are not kept). Regrowing a
// buffer drops the captured batch graph, which may reference it.
cudaError_t ensure_buffer(FjCuda* cuda, float*& buf, size_t& have, size_t bytes) {
    if (have >= bytes && buf) return cudaSuccess;
    if (buf) {
        batch_graph_release(cuda);
        cudaFree(buf);
    }
    buf = nullptr;
    have = 0;
    cudaError_t e = cudaMalloc(&buf, bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}

void stage_begin(FjCuda* cuda, int stage, void* vs) {
    if (!cuda->timing || !cuda->timing_events) return;
    cudaEventRecord(cuda->stage_ev[2 * stage], reinterpret_cast<cudaStream_t>(vs));
    cuda->stage_open[stage] = true;
}

void stage_end(FjCuda* cuda, int stage, void* vs) {
    if (!cuda->timing || !cuda->timing_events || !cuda->stage_open[stage]) return;
    cudaEventRecord(cuda->stage_ev[2 * stage + 1], reinterpret_cast<cudaStream_t>(vs));
}

// After the frame's stream has drained: fold the recorded stage intervals into the totals.
void stage_collect(FjCuda* cuda) {
    for (int s = 0; s < FJB_STAGE_COUNT; ++s) {
        if (!cuda->stage_open[s]) continue;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, cuda->stage_ev[2 * s], cuda->stage_ev[2 * s + 1]) == cudaSuccess) {
            cuda->stage_ms[s] += ms;
            cuda->stage_frames[s] += 1;
        }
        cuda->stage_open[s] = false;
    }
}

void stage_events_release(FjCuda* cuda) {
    if (!cuda->timing_events) return;
    for (cudaEvent_t& e : cuda->stage_ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    cuda->timing_events = false;
}

// FNV-1a over the bytes of individual fields: identities of descriptor contents for
// the owner's caches (never of padding).
struct Fnv {
    uint64_t h = 0xcbf29ce484222325ULL;
    template <typename T>
    Fnv& add(const T& v) {
        const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
        for (size_t i = 0; i < sizeof(T); ++i) {
            h ^= b[i];
            h *= 0x100000001b3ULL;
        }
        return *this;
    }
};

uint64_t diffusion_identity(const FjDiffusion& d) {
    Fnv f;
    f.add(d.family).add(d.scatter_fraction).add(d.warmth).add(d.spatial_scale).add(d.pixel_size_um).add(d.radius_px);
    for (int i = 0; i < 3; ++i) f.add(d.group_weights[i]).add(d.group_lambda_um[i]);
    return f.h | 1;
}

uint64_t spatial_dir_identity(const FjSpatialDir& sd, int width, int height) {
    Fnv f;
    f.add(width).add(height).add(sd.component_count);
    for (const FjExtent* e : {&sd.render_extent, &sd.full_frame_extent, &sd.filter_domain_extent})
        f.add(e->x).add(e->y).add(e->width).add(e->height);
    for (size_t k = 0; k < sd.component_count && k < 4; ++k) {
        const FjDirGaussian& g = sd.components[k];
        f.add(g.sigma_px).add(g.weight).add(g.radius).add(g.reference_operator).add(g.feedforward);
        for (int i = 0; i < 3; ++i) f.add(g.feedback[i]).add(g.feedback_numerators[i]);
        f.add(g.normalization_denominator).add(g.feedforward_numerator).add(g.boundary_truncation_accuracy);
        f.add(g.boundary_certification_tolerance).add(g.boundary_derivation_version);
    }
    return f.h | 1;
}

bool same_rect(const FjRect& a, const FjRect& b) { return a.x1 == b.x1 && a.y1 == b.y1 && a.x2 == b.x2 && a.y2 == b.y2; }

// Stages this build schedules; the others are rejected by name rather than skipped.
bool stages_supported(const FjPreparedHostData& h, std::string& why) {
    // the reference admits enlarger diffusion on the print routes only
    // (native/juicer_cuda_descriptors.cpp:206-216)
    if ((h.optics.flags & FJ_OPTICS_ENLARGER_DIFFUSION) && h.route != FJ_ROUTE_NEGATIVE_PRINT &&
        h.route != FJ_ROUTE_POSITIVE_PRINT) {
        why = "invalid descriptor: optics.flags (enlarger diffusion needs a print route)";
        return false;
    }
    fjb::PostPlan post;
    if (!fjb::post_plan_from(h.scanner_post, post, why)) return false;
    fjb::EffectsPlan effects;
    if (!fjb::effects_plan_from(h.effects, effects, why)) return false;
    return true;
}

cudaError_t ensure_scalar(FjCuda* cuda) {
    if (cuda->ae_scale) return cudaSuccess;
    return cudaMalloc(&cuda->ae_scale, 256);
}

cudaError_t ensure_work(FjCuda* cuda, size_t bytes) {
    if (cuda->work_bytes >= bytes) return cudaSuccess;
    batch_graph_release(cuda);
    if (cuda->work) cudaFree(cuda->work);
    cuda->work = nullptr;
    cuda->work_bytes = 0;
    cudaError_t e = cudaMalloc(&cuda->work, bytes);
    if (e == cudaSuccess) cuda->work_bytes = bytes;
    return e;
}

// Device copy of the static grain noise, uploaded once per distinct host buffer.
FjStatus ensure_noise(FjCuda* cuda, const FjStaticNoise& n, void* stream, const FjbNoise** out, FjErrorBuffer* error) {
    *out = nullptr;
    if (!n.stbn.data || n.stbn.count == 0) return fjb::ok_status();
    const uintptr_t k0 = reinterpret_cast<uintptr_t>(n.stbn.data), k1 = reinterpret_cast<uintptr_t>(n.wang_tiles.data);
    if (cuda->noise && cuda->noise_key[0] == k0 && cuda->noise_key[1] == k1 && cuda->noise_key[2] == n.stbn.count) {
        *out = cuda->noise;
        return fjb::ok_status();
    }
    if (cuda->noise) {
        fjb_noise_destroy(cuda->noise, nullptr);
        cuda->noise = nullptr;
    }
    FjbNoise* fresh = nullptr;
    FjStatus st = fjb_noise_create(&n, stream, &fresh, error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    cuda->noise = fresh;
    cuda->noise_key[0] = k0;
    cuda->noise_key[1] = k1;
    cuda->noise_key[2] = n.stbn.count;
    *out = fresh;
    return fjb::ok_status();
}

// One diffusion stage (camera or enlarger, src/Cuda/Diffusion/JuicerCudaDiffusion.cu:779
// launch_stage) from planes R, G, B `src` into `dst`: PSF rows built once per descriptor,
// FFT form from radius 8 up (PSF spectrum once per descriptor and frame size), else the
// direct form. Times the launch as `stage`.
// Key of a diffusion form decision: the frame size and radius.
uint64_t diffusion_form_key(int width, int height, int radius) {
    Fnv f;
    f.add(width).add(height).add(radius);
    return f.h | 1;
}

FjStatus apply_diffusion(FjCuda* cuda, const FjDiffusion& d, int stage, const float* src[3], float* dst[3],
                         ptrdiff_t stride, int width, int height, void* vs, FjErrorBuffer* error) {
    if (!(d.scatter_fraction >= 0.0 && d.scatter_fraction <= 1.0))
        return fjb::fail_status(FJ_STATUS_PREPARATION_FAILURE, error, "diffusion scatter fraction outside [0, 1]");
    cudaError_t e = cudaSuccess;
    const uint64_t key = diffusion_identity(d);
    Fnv ck;
    ck.add(stage).add(key).add(width).add(height);
    auto found = cuda->diffusion.find(ck.h);
    if (found == cuda->diffusion.end()) {
        cache_room(cuda, cuda->diffusion);
        found = cuda->diffusion.emplace(ck.h, fjb_sched::DiffusionCache{}).first;
    }
    fjb_sched::DiffusionCache& cache = found->second;
    if (key != cache.key || !cache.psf) {
        // PSF rows are built once per distinct descriptor and kept on the device
        FjDiffusionComponents dc{};
        FjStatus st = fjb_diffusion_components_host(&d, &dc, error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        const double* wts[3] = {dc.red_weights, dc.green_weights, dc.blue_weights};
        std::vector<float> rows[3];
        int taps = 0;
        std::string why;
        for (int c = 0; c < 3; ++c)
            if (!fjb::diffusion_psf_rows(dc.lambda_px, wts[c], d.radius_px, rows[c], taps, why))
                return fjb::fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
        const size_t bytes = 3 * rows[0].size() * sizeof(float);
        cache.key = 0;
        e = ensure_buffer(cuda, cache.psf, cache.psf_bytes, bytes);
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "diffusion PSF");
        for (int c = 0; c < 3 && e == cudaSuccess; ++c)
            e = cudaMemcpy(cache.psf + c * rows[0].size(), rows[c].data(), rows[c].size() * sizeof(float),
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "diffusion PSF upload");
        cache.key = key;
        cache.taps = taps;
    }
    const size_t n = (size_t)(d.radius_px + 1) * (size_t)cache.taps;
    const float* psf[3] = {cache.psf, cache.psf + n, cache.psf + 2 * n};
    const cudaStream_t cs = reinterpret_cast<cudaStream_t>(vs);
    fjb::DiffusionFftPlan plan;
    const bool fft_possible = fjb::diffusion_fft_plan(width, height, d.radius_px, plan);
    // the form: the owner's measured choice when autotuning, else the fixed rule
    const uint64_t fkey = diffusion_form_key(width, height, d.radius_px);
    const auto decided = cuda->diffusion_form.find(fkey);
    const bool measure = cuda->autotune && !cuda->capturing && fft_possible && decided == cuda->diffusion_form.end();
    bool fft = fft_possible && fjb::diffusion_prefers_fft(width, height, d.radius_px);
    if (cuda->autotune && decided != cuda->diffusion_form.end()) fft = fft_possible && decided->second == FJB_DIFFUSION_FFT;
    if (fft || measure) {
        // the PSF spectrum depends on the descriptor and the transform sizes
        const uint64_t skey = (cache.key * 0x100000001b3ULL) ^ ((uint64_t)width << 32) ^ (uint64_t)height;
        e = ensure_buffer(cuda, cuda->diffusion_fft_work, cuda->diffusion_fft_work_bytes,
                          plan.work_floats * sizeof(float));
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "diffusion FFT workspace");
        if (skey != cache.spectrum_key || !cache.spectrum) {
            cache.spectrum_key = 0;
            e = ensure_buffer(cuda, cache.spectrum, cache.spectrum_bytes, plan.spectrum_floats * sizeof(float));
            if (e != cudaSuccess) return fjb::cuda_status(e, error, "diffusion PSF spectrum");
            e = fjb::launch_diffusion_fft_spectrum(plan, psf, cache.taps, cache.spectrum, cuda->diffusion_fft_work, cs);
            if (e != cudaSuccess) return fjb::cuda_status(e, error, "diffusion PSF spectrum");
            cache.spectrum_key = skey;
        }
    }
    auto run = [&](bool use_fft) {
        return use_fft ? fjb::launch_diffusion_fft(plan, cache.spectrum, (float)d.scatter_fraction, dst, src, stride,
                                                   cuda->diffusion_fft_work, cs)
                       : fjb::launch_diffusion(psf, d.radius_px, cache.taps, (float)d.scatter_fraction, dst, src,
                                               stride, width, height, cs);
    };
    if (measure) {
        // time both forms on this frame's planes (second of two runs each), keep the faster
        cudaEvent_t a = nullptr, b = nullptr;
        float ms[2] = {0.0f, 0.0f};
        e = cudaEventCreate(&a);
        if (e == cudaSuccess) e = cudaEventCreate(&b);
        for (int f = 0; f < 2 && e == cudaSuccess; ++f) {
            e = run(f == 1);
            if (e == cudaSuccess) e = cudaEventRecord(a, cs);
            if (e == cudaSuccess) e = run(f == 1);
            if (e == cudaSuccess) e = cudaEventRecord(b, cs);
            if (e == cudaSuccess) e = cudaEventSynchronize(b);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[f], a, b);
        }
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "diffusion form measurement");
        fft = ms[1] < ms[0];
        if (cuda->diffusion_form.size() >= fjb_sched::kCacheEntries) cuda->diffusion_form.clear();
        cuda->diffusion_form[fkey] = fft ? FJB_DIFFUSION_FFT : FJB_DIFFUSION_DIRECT;
    }
    stage_begin(cuda, stage, vs);
    e = run(fft);
    stage_end(cuda, stage, vs);
    if (e != cudaSuccess) return fjb::cuda_status(e, error, "diffusion");
    return fjb::ok_status();
}

// The staged schedule of src/Cuda/JuicerCudaExecutor.cpp:1874-2400: camera exposure
// to carrier planes, camera diffusion, scatter/halation, spatial DIR, capture
// density, grain, then print/scan/output from the density planes.
FjStatus render_staged(FjCuda* cuda, FjbRecipe* recipe, const FjPreparedHostData& h, const float* src, ptrdiff_t srb,
                       float* dst, ptrdiff_t drb, int width, int height, uint32_t comps, void* vs,
                       const FjAbortCallback& abort_cb, bool camera_diffusion, bool halation, bool spatial_dir,
                       bool grain, const fjb::PostPlan& post, const fjb::EffectsPlan& fx, uint64_t glare_seed,
                       int glare_x, int glare_y, void* boost_state, FjErrorBuffer* error) {
    const size_t plane = (size_t)width * (size_t)height;
    const size_t plane_bytes = (plane * sizeof(float) + 255) / 256 * 256;
    // linear planes before the encoding: scanner post effects or film / gate defects
    const bool planes_out = post.active || fx.film || fx.gate_output;
    size_t scratch = 0;
    if (planes_out) scratch = std::max(scratch, fjb_scanner_post_scratch_bytes(width, height));
    if (halation) scratch = std::max(scratch, fjb_scatter_halation_scratch_bytes(width, height));
    if (spatial_dir) scratch = std::max(scratch, fjb_spatial_dir_scratch_bytes(width, height));
    if (grain) scratch = std::max(scratch, fjb_visual_grain_scratch_bytes(width, height));
    const int planes = 3 + 3 + (spatial_dir ? 6 : 0) + (fx.film_dust ? 1 : 0);
    const size_t mask_bytes =
        fx.gate_mask ? ((size_t)h.effects.gate_width * (size_t)h.effects.gate_height * sizeof(float) + 255) / 256 * 256
                     : 0;
    // the defect particle tables (film families, then gate families, in turn)
    const size_t table_bytes = std::max(fx.film ? fjb::film_defects_table_bytes(h.effects, width, height) : 0,
                                        fx.gate_mask ? fjb::gate_mask_table_bytes(h.effects, h.effects.gate_width,
                                                                                  h.effects.gate_height)
                                                     : 0);
    cudaError_t e = ensure_work(cuda, planes * plane_bytes + scratch + mask_bytes + table_bytes + 256);
    FjStatus st{};
    if (e != cudaSuccess) return fjb::cuda_status(e, error, "frame workspace");
    char* base = static_cast<char*>(cuda->work);
    auto P = [&](int i) { return reinterpret_cast<float*>(base + (size_t)i * plane_bytes); };
    float* carrier[3] = {P(0), P(1), P(2)}; // B, G, R
    float* density[3] = {P(3), P(4), P(5)}; // C, M, Y (also the diffusion target)
    float* dirp[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (spatial_dir)
        for (int i = 0; i < 6; ++i) dirp[i] = P(6 + i);
    float* dust = fx.film_dust ? P(planes - 1) : nullptr;
    float* scratch_p = reinterpret_cast<float*>(base + (size_t)planes * plane_bytes);
    float* gate_mask = fx.gate_mask ? reinterpret_cast<float*>(base + (size_t)planes * plane_bytes + scratch) : nullptr;
    void* tables = table_bytes ? base + (size_t)planes * plane_bytes + scratch + mask_bytes : nullptr;
    const ptrdiff_t stride = width;
    const FjOptics& o = h.optics;

    stage_begin(cuda, FJB_STAGE_CAMERA_EXPOSURE, vs);
    st = fjb_camera_exposure(recipe, src, srb, comps, width, height, carrier[0], carrier[1], carrier[2], stride, vs,
                             error);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (aborted(abort_cb)) return fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
    if (o.flags & FJ_OPTICS_HIGHLIGHT_BOOST) {
        // highlight reconstruction on the carrier, before diffusion; the disposition is
        // checked when the frame's flags are read
        if (!boost_state) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "highlight boost state missing");
        st = fjb_highlight_boost(&o.highlight_boost, carrier[0], carrier[1], carrier[2], stride, width, height,
                                 boost_state, vs, error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
    }
    stage_end(cuda, FJB_STAGE_CAMERA_EXPOSURE, vs);
    if (camera_diffusion) {
        // R, G, B carrier planes into the density planes, which then carry the exposure
        float* ddst[3] = {density[2], density[1], density[0]};
        const float* dsrc[3] = {carrier[2], carrier[1], carrier[0]};
        st = apply_diffusion(cuda, o.camera, FJB_STAGE_CAMERA_DIFFUSION, dsrc, ddst, stride, width, height, vs,
                             error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        std::swap(carrier[0], density[0]);
        std::swap(carrier[1], density[1]);
        std::swap(carrier[2], density[2]);
        if (aborted(abort_cb)) return fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
    }
    if (halation) {
        stage_begin(cuda, FJB_STAGE_SCATTER_HALATION, vs);
        st = fjb_scatter_halation(&o.scatter_halation, carrier[2], carrier[1], carrier[0], stride, width, height,
                                  scratch_p, scratch, vs, error);
        stage_end(cuda, FJB_STAGE_SCATTER_HALATION, vs);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        if (aborted(abort_cb)) return fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
    }
    if (spatial_dir) {
        const uint64_t key = spatial_dir_identity(h.spatial_dir, width, height);
        auto found = cuda->dir_plans.find(key);
        if (found == cuda->dir_plans.end()) {
            // operator tables (taps, reflected boundaries) are built once per geometry
            cache_room(cuda, cuda->dir_plans);
            fjb::DirPlan fresh;
            std::string why;
            e = cudaSuccess;
            if (!fjb::dir_plan_create(h.spatial_dir, width, height, reinterpret_cast<cudaStream_t>(vs), fresh, why, e)) {
                fresh.release();
                if (e != cudaSuccess) return fjb::cuda_status(e, error, "spatial DIR plan");
                return fjb::fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
            }
            found = cuda->dir_plans.emplace(key, std::move(fresh)).first;
        }
        stage_begin(cuda, FJB_STAGE_SPATIAL_DIR, vs);
        st = fjb::spatial_dir_apply(recipe, found->second, nullptr, 0, 3, carrier[0], carrier[1], carrier[2], stride,
                                    width, height, dirp[0], dirp[1], dirp[2], dirp[3], dirp[4], dirp[5], scratch_p,
                                    scratch, vs, error);
        stage_end(cuda, FJB_STAGE_SPATIAL_DIR, vs);
        if (st.category == FJ_STATUS_SUCCESS)
            st = fjb_recipe_set_spatial_dir_planes(recipe, dirp[0], dirp[1], dirp[2], dirp[3], dirp[4], dirp[5], error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        if (aborted(abort_cb)) return fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
    }
    stage_begin(cuda, FJB_STAGE_CAPTURE_DENSITY, vs);
    st = fjb_capture_density(recipe, nullptr, 0, 3, carrier[0], carrier[1], carrier[2], stride, width, height,
                             density[0], density[1], density[2], vs, error);
    stage_end(cuda, FJB_STAGE_CAPTURE_DENSITY, vs);
    if (st.category != FJ_STATUS_SUCCESS) return st;
    if (grain) {
        const FjVisualGrain& g = h.grain;
        if (g.render_extent.width != width || g.render_extent.height != height)
            return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "grain render extent differs from the render window");
        const FjbNoise* noise = nullptr;
        st = ensure_noise(cuda, h.noise, vs, &noise, error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        stage_begin(cuda, FJB_STAGE_GRAIN, vs);
        st = fjb_visual_grain(recipe, &g, noise, density[0], density[1], density[2], stride, width, height, scratch_p,
                              scratch, vs, error);
        stage_end(cuda, FJB_STAGE_GRAIN, vs);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        if (aborted(abort_cb)) return fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
    }
    if (fx.film) {
        // film dust and scratches on the developed capture density, after grain
        // (src/Cuda/JuicerCudaExecutor.cpp:1674-1690, :2263-2279)
        stage_begin(cuda, FJB_STAGE_FILM_DEFECTS, vs);
        e = fjb::launch_film_defects(h.effects, width, height, density[0], density[1], density[2], dust,
                                     reinterpret_cast<cudaStream_t>(vs), tables, table_bytes);
        stage_end(cuda, FJB_STAGE_FILM_DEFECTS, vs);
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "film defects");
    }
    // Enlarger diffusion (src/Cuda/JuicerCudaExecutor.cpp:2292-2365): the print-linear
    // exposure of the capture density (film dust applied there) into the carrier planes,
    // the enlarger's diffusion back into the density planes, print development there;
    // the scan then reads print density and the film dust is not applied again.
    const bool enlarger = (o.flags & FJ_OPTICS_ENLARGER_DIFFUSION) != 0;
    if (enlarger) {
        st = fjb_enlarger_linear_exposure(recipe, density[0], density[1], density[2], dust, carrier[0], carrier[1],
                                          carrier[2], width, height, vs, error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        const float* dsrc[3] = {carrier[0], carrier[1], carrier[2]}; // red-, green-, blue-sensitive layers
        float* ddst[3] = {density[0], density[1], density[2]};
        st = apply_diffusion(cuda, o.enlarger, FJB_STAGE_ENLARGER_DIFFUSION, dsrc, ddst, stride, width, height, vs,
                             error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        st = fjb_enlarger_develop(recipe, density[0], density[1], density[2], density[0], density[1], density[2],
                                  width, height, vs, error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        dust = nullptr;
        recipe->r.params.print_done = 1;
        if (aborted(abort_cb)) return fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
    }
    if (planes_out) {
        fjb::OutputEffects out;
        out.dust = dust;
        if (fx.gate_output) {
            const FjFilmEffects& fe = h.effects;
            out.weave = fx.weave;
            out.weave_dx = fe.weave_dx_px;
            out.weave_dy = fe.weave_dy_px;
            out.weave_cos = fe.weave_cos_rot;
            out.weave_sin = fe.weave_sin_rot;
            out.roi_x = fe.roi_offset_x;
            out.roi_y = fe.roi_offset_y;
            if (fx.gate_mask) {
                // gate dust and scratches at the gate grid (src/Cuda/JuicerCudaExecutor.cpp:2788-2790)
                e = fjb::launch_gate_mask(fe, gate_mask, fe.gate_width, fe.gate_height,
                                          reinterpret_cast<cudaStream_t>(vs), tables, table_bytes);
                if (e != cudaSuccess) return fjb::cuda_status(e, error, "gate mask");
                out.gate_mask = gate_mask;
                out.gate_w = fe.gate_width;
                out.gate_h = fe.gate_height;
            }
        }
        // scanner post effects: taps kept on the device per descriptor (keyed by its
        // hash and the taps' length)
        const std::vector<float> taps = fjb::post_taps(post);
        const uint64_t tkey = (h.scanner_post.hash * 0x100000001b3ULL) ^ (uint64_t)taps.size();
        auto tap = cuda->post_taps.find(tkey);
        if (tap == cuda->post_taps.end()) {
            cache_room(cuda, cuda->post_taps);
            tap = cuda->post_taps.emplace(tkey, fjb_sched::DeviceFloats{}).first;
            if (!taps.empty()) {
                e = ensure_buffer(cuda, tap->second.data, tap->second.bytes, taps.size() * sizeof(float));
                if (e == cudaSuccess)
                    e = cudaMemcpy(tap->second.data, taps.data(), taps.size() * sizeof(float), cudaMemcpyHostToDevice);
                if (e != cudaSuccess) {
                    tap->second.release();
                    cuda->post_taps.erase(tap);
                    return fjb::cuda_status(e, error, "scanner post taps");
                }
            }
        }
        stage_begin(cuda, FJB_STAGE_PRINT_SCAN_OUTPUT, vs);
        st = fjb::render_from_density_post(recipe, post, glare_seed, glare_x, glare_y, density[0], density[1],
                                           density[2], comps == 4 ? src : nullptr, srb, dst, drb, width, height, comps,
                                           scratch_p, tap->second.data, reinterpret_cast<cudaStream_t>(vs), error,
                                           out);
        stage_end(cuda, FJB_STAGE_PRINT_SCAN_OUTPUT, vs);
        return st;
    }
    stage_begin(cuda, FJB_STAGE_PRINT_SCAN_OUTPUT, vs);
    st = fjb_render_from_density(recipe, density[0], density[1], density[2], comps == 4 ? src : nullptr, srb, dst, drb,
                                 width, height, comps, vs, error);
    stage_end(cuda, FJB_STAGE_PRINT_SCAN_OUTPUT, vs);
    return st;
}

// ---------------------------------------------------------------------------
// One frame, in three steps shared by fj_cuda_render and fjb_render_batch: the
// admission checks (host only), the enqueue of its work on a stream, and its outcome
// from the flag word the frame left.
// ---------------------------------------------------------------------------
struct FrameWork {
    FjbRecipe* recipe = nullptr;
    std::unique_ptr<FjbRecipe> transient; // recipe_hash 0: this frame's own tables
    bool boost = false;
    void* boost_state = nullptr;
    ~FrameWork() {
        if (transient) transient->r.release();
    }
};

FjStatus frame_check(FjCuda* cuda, const FjCudaContext* context, const FjFrame* frame,
                     const FjPreparedHostData* prepared, FjErrorBuffer* error) {
    (void)cuda;
    int dev = 0;
    cudaGetDevice(&dev);
    if (context->device_id != dev)
        return fjb::fail_status(FJ_STATUS_CONTEXT_LOSS, error, "current device differs from the inspected one");
    if (!image_ok(frame->source) || !image_ok(frame->destination) ||
        frame->source.components != frame->destination.components ||
        !rect_inside(frame->render_window, frame->source.bounds) ||
        !rect_inside(frame->render_window, frame->destination.bounds))
        return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "frame images or render window rejected");
    const uint32_t optics = prepared->optics.flags;
    if (optics != 0 && (!same_rect(frame->source.bounds, frame->full_frame_extent) ||
                        !same_rect(frame->destination.bounds, frame->full_frame_extent) ||
                        !same_rect(frame->render_window, frame->full_frame_extent)))
        return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "CUDA optics require the complete frame domain");
    // a weave-carrying effects record needs the complete frame domain, as the optics
    // do (src/Cuda/JuicerCudaExecutor.cpp:752-768)
    if ((prepared->effects.flags & FJ_EFFECTS_FULL_FRAME) != 0 &&
        (prepared->effects.flags & (FJ_EFFECTS_FILM | FJ_EFFECTS_GATE_OUTPUT)) != 0 &&
        (!same_rect(frame->source.bounds, frame->full_frame_extent) ||
         !same_rect(frame->destination.bounds, frame->full_frame_extent) ||
         !same_rect(frame->render_window, frame->full_frame_extent)))
        return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "film effects require the complete frame domain");
    std::string unsupported;
    if (!stages_supported(*prepared, unsupported)) return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, unsupported);
    if ((prepared->film_exposure.flags & FJ_FILM_AUTO_EXPOSURE) &&
        !rect_inside(prepared->auto_exposure.source_bounds, frame->source.bounds))
        return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error,
                                "auto exposure source bounds outside the source image");
    return fjb::ok_status();
}

// Enqueues a checked frame on `stream`. With highlight reconstruction the frame's
// maximum and disposition go to `boost_state`. Frame-scoped recipe state (the
// auto-exposure scale pointer, the print-done mark, the spatial-DIR planes) is reset
// when this returns: the launches have taken their parameters by then.
FjStatus frame_enqueue(FjCuda* cuda, const FjFrame* frame, const FjSubmission* submission,
                       const FjPreparedHostData* prepared, const FjAbortCallback& abort_callback, cudaStream_t stream,
                       void* boost_state, FrameWork& work, FjErrorBuffer* error) {
    void* vs = reinterpret_cast<void*>(stream);
    int dev = 0;
    cudaGetDevice(&dev);
    // ---- recipe tables (cached by recipe_hash; hash 0 = this frame only) ----
    FjbRecipe* recipe = nullptr;
    const uint64_t key = prepared->recipe_hash;
    if (key != 0) {
        auto it = cuda->recipes.find(key);
        if (it != cuda->recipes.end()) recipe = it->second;
    }
    if (!recipe) {
        std::unique_ptr<FjbRecipe> fresh(new FjbRecipe());
        fresh->device = dev;
        std::string why;
        FjStatus st{};
        if (!fjb::create_recipe(*prepared, stream, fresh->r, why, st)) {
            fjb::write_error(error, why);
            return st;
        }
        recipe = fresh.get();
        if (key != 0)
            cuda->recipes[key] = fresh.release();
        else
            work.transient = std::move(fresh);
    }
    work.recipe = recipe;
    recipe->r.params.print_form = cuda->print_form;
    struct FrameState {
        FjbRecipe* r;
        ~FrameState() {
            r->r.params.auto_exposure_scale = nullptr;
            r->r.params.print_done = 0;
            fjb_recipe_set_spatial_dir_planes(r, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        }
    } frame_state{recipe};

    const FjRect& w = frame->render_window;
    const int width = w.x2 - w.x1, height = w.y2 - w.y1;
    const uint32_t comps = frame->source.components;
    const float* src = reinterpret_cast<const float*>(pixel_address(frame->source, w.x1, w.y1));
    float* dst = const_cast<float*>(reinterpret_cast<const float*>(pixel_address(frame->destination, w.x1, w.y1)));
    const ptrdiff_t srb = frame->source.row_bytes, drb = frame->destination.row_bytes;
    FjStatus st = fjb_recipe_clear_flags(recipe, vs, error);
    if (st.category != FJ_STATUS_SUCCESS) return st;

    // ---- camera auto exposure (src/Cuda/JuicerCudaExecutor.cpp:1013) ----
    if (prepared->film_exposure.flags & FJ_FILM_AUTO_EXPOSURE) {
        const FjAutoExposure& ae = prepared->auto_exposure;
        cudaError_t e = ensure_scalar(cuda);
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "auto exposure scale");
        const float* msrc =
            reinterpret_cast<const float*>(pixel_address(frame->source, ae.source_bounds.x1, ae.source_bounds.y1));
        stage_begin(cuda, FJB_STAGE_AUTO_EXPOSURE, vs);
        st = fjb_auto_exposure(recipe, msrc, srb, comps, &ae, cuda->ae_scale, vs, error);
        stage_end(cuda, FJB_STAGE_AUTO_EXPOSURE, vs);
        if (st.category == FJ_STATUS_SUCCESS) st = fjb_recipe_set_exposure_scale_device(recipe, cuda->ae_scale, error);
        if (st.category != FJ_STATUS_SUCCESS) return st;
    }

    const uint32_t optics = prepared->optics.flags;
    const bool camera_diffusion = (optics & FJ_OPTICS_CAMERA_DIFFUSION) != 0;
    const bool halation = (optics & FJ_OPTICS_SCATTER_HALATION) != 0;
    const bool spatial_dir = prepared->spatial_dir.component_count > 0;
    const bool grain = (prepared->grain.flags & FJ_GRAIN_ACTIVE) != 0;
    fjb::PostPlan post;
    fjb::EffectsPlan fx;
    {
        std::string why;
        if (!fjb::post_plan_from(prepared->scanner_post, post, why) || !fjb::effects_plan_from(prepared->effects, fx, why))
            return fjb::fail_status(FJ_STATUS_PREPARATION_FAILURE, error, why);
    }
    work.boost = (optics & FJ_OPTICS_HIGHLIGHT_BOOST) != 0;
    work.boost_state = boost_state;
    const bool enlarger = (optics & FJ_OPTICS_ENLARGER_DIFFUSION) != 0;
    if (!camera_diffusion && !halation && !spatial_dir && !grain && !post.active && !work.boost && !fx.film &&
        !fx.gate_output && !enlarger) {
        // Monolithic: one fused pass source -> output
        stage_begin(cuda, FJB_STAGE_MONOLITHIC, vs);
        st = fjb_render_pixels(recipe, src, srb, dst, drb, width, height, comps, vs, error);
        stage_end(cuda, FJB_STAGE_MONOLITHIC, vs);
        return st;
    }
    // the glare noise is keyed by the recipe, the frame token and the source origin
    // (src/Cuda/JuicerCudaExecutor.cpp:2416-2420)
    const uint64_t seed = fjb::glare_seed(prepared->recipe_hash, submission ? submission->frame_token : 0,
                                          frame->source.bounds.x1, frame->source.bounds.y1);
    return render_staged(cuda, recipe, *prepared, src, srb, dst, drb, width, height, comps, vs, abort_callback,
                         camera_diffusion, halation, spatial_dir, grain, post, fx, seed, frame->source.bounds.x1,
                         frame->source.bounds.y1, boost_state, error);
}

// The outcome of an enqueued frame from its flag word (after the stream has drained).
FjRenderOutcome frame_outcome(FrameWork& work, uint32_t flags, cudaStream_t stream, FjErrorBuffer* error) {
    FjRenderOutcome out{};
    if (work.boost) {
        // src/ProcessRoot.cpp:4063-4096: an invalid carrier or peak overflow fails the frame
        FjStatus st = fjb_highlight_boost_result(work.boost_state, reinterpret_cast<void*>(stream), nullptr, error);
        if (st.category != FJ_STATUS_SUCCESS) {
            out.status = st;
            return out;
        }
    }
    if (flags & fjb::kErrTensorWait) {
        out.status = fjb::fail_status(FJ_STATUS_CUDA_FAILURE, error,
                                      "print stage: a tensor-core completion wait ran out of time");
        return out;
    }
    if (flags & (1u << 8)) out.flags |= FJ_RENDER_DEFERRED_DIR_ERROR;
    out.status = fjb::ok_status();
    fjb::write_error(error, (flags & 1u) ? "scanner stage reported non-finite pixels" : "");
    return out;
}

cudaError_t ensure_boost(void*& state) {
    if (state) return cudaSuccess;
    return cudaMalloc(&state, fjb_highlight_boost_state_bytes());
}

} // namespace

extern "C" {

FjStatus fj_cuda_create(FjCuda** out_cuda, FjErrorBuffer* error) {
    try {
        if (!out_cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "out_cuda is null");
        *out_cuda = nullptr;
        auto* owner = new (std::nothrow) FjCuda();
        if (!owner) return fjb::fail_status(FJ_STATUS_ALLOCATION_FAILURE, error, "owner allocation failed");
        FjCuda* expected = nullptr;
        if (!g_live_owner.compare_exchange_strong(expected, owner)) {
            delete owner;
            return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "a live FjCuda owner already exists");
        }
        *out_cuda = owner;
        fjb::write_error(error, "");
        return fjb::ok_status();
    } catch (...) {
        return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fj_cuda_create");
    }
}

FjStatus fj_cuda_check_terminal(FjCuda* cuda, FjErrorBuffer* error) {
    if (!cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null owner");
    std::lock_guard<std::mutex> lock(cuda->gate);
    if (cuda->closed) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fj_cuda_inspect(FjCuda* cuda, const FjFrame* frame, FjCudaContext* out_context, FjErrorBuffer* error) {
    try {
        if (!cuda || !frame || !out_context) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        std::lock_guard<std::mutex> lock(cuda->gate);
        if (cuda->closed) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
        if (!image_ok(frame->source) || !image_ok(frame->destination))
            return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error,
                                    "images must be float32 RGB/RGBA device buffers with valid bounds");
        if (frame->source.components != frame->destination.components)
            return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "source/destination component mismatch");
        if (!rect_inside(frame->render_window, frame->source.bounds) ||
            !rect_inside(frame->render_window, frame->destination.bounds))
            return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "render window outside image bounds");
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "cudaGetDevice");
        out_context->device_id = dev;
        out_context->context = 0;
        fjb::write_error(error, "");
        return fjb::ok_status();
    } catch (...) {
        return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fj_cuda_inspect");
    }
}

FjRenderOutcome fj_cuda_render(FjCuda* cuda, const FjCudaContext* context, const FjFrame* frame,
                               const FjSubmission* submission, const FjPreparedHostData* prepared,
                               FjAbortCallback abort_callback, FjErrorBuffer* error) {
    FjRenderOutcome out{};
    try {
        if (!cuda || !context || !frame || !prepared) {
            out.status = fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
            return out;
        }
        std::lock_guard<std::mutex> lock(cuda->gate);
        if (cuda->closed) {
            out.status = fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
            return out;
        }
        FjStatus st = frame_check(cuda, context, frame, prepared, error);
        if (st.category != FJ_STATUS_SUCCESS) {
            out.status = st;
            return out;
        }
        if (aborted(abort_callback)) {
            out.status = fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
            return out;
        }
        const bool hostStream = (frame->flags & FJ_FRAME_STREAM_PRESENT) != 0;
        cudaStream_t stream = hostStream ? reinterpret_cast<cudaStream_t>(frame->stream) : nullptr;
        void* boost = nullptr;
        if (prepared->optics.flags & FJ_OPTICS_HIGHLIGHT_BOOST) {
            const cudaError_t e = ensure_boost(cuda->boost_state);
            if (e != cudaSuccess) {
                out.status = fjb::cuda_status(e, error, "highlight boost state");
                return out;
            }
            boost = cuda->boost_state;
        }
        FrameWork work;
        st = frame_enqueue(cuda, frame, submission, prepared, abort_callback, stream, boost, work, error);
        if (st.category != FJ_STATUS_SUCCESS) {
            cudaStreamSynchronize(stream);
            for (bool& o : cuda->stage_open) o = false;
            out.status = st;
            return out;
        }
        uint32_t flags = 0;
        st = fjb_recipe_read_flags(work.recipe, reinterpret_cast<void*>(stream), &flags, error);
        if (st.category != FJ_STATUS_SUCCESS) {
            out.status = st;
            return out;
        }
        stage_collect(cuda);
        return frame_outcome(work, flags, stream, error);
    } catch (...) {
        out.status = fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fj_cuda_render");
        return out;
    }
}

FjStatus fjb_render_batch(FjCuda* cuda, const FjCudaContext* context, const FjFrame* frames,
                          const FjSubmission* submissions, const FjPreparedHostData* const* prepared, int32_t count,
                          void* stream, uint64_t graph_token, FjRenderOutcome* outcomes, FjErrorBuffer* error) {
    try {
        if (!cuda || !context || !frames || !prepared || !outcomes || count < 0)
            return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        std::lock_guard<std::mutex> lock(cuda->gate);
        if (cuda->closed) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
        for (int32_t i = 0; i < count; ++i) outcomes[i] = FjRenderOutcome{};
        bool transient = false;
        for (int32_t i = 0; i < count; ++i) {
            if (!prepared[i]) {
                outcomes[i].status = fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
                return outcomes[i].status;
            }
            outcomes[i].status = frame_check(cuda, context, &frames[i], prepared[i], error);
            if (outcomes[i].status.category != FJ_STATUS_SUCCESS) return outcomes[i].status;
            transient = transient || prepared[i]->recipe_hash == 0;
        }
        if (count == 0) {
            fjb::write_error(error, "");
            return fjb::ok_status();
        }
        const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        // a graph needs a capturable stream and recipes that outlive the call
        const bool graph = graph_token != 0 && s != nullptr && !transient;
        cudaError_t e = cudaSuccess;
        if (cuda->batch_slots < (size_t)count) {
            batch_graph_release(cuda);
            if (cuda->batch_flags) cudaFree(cuda->batch_flags);
            if (cuda->batch_flags_host) cudaFreeHost(cuda->batch_flags_host);
            cuda->batch_flags = nullptr;
            cuda->batch_flags_host = nullptr;
            cuda->batch_slots = 0;
            e = cudaMalloc(&cuda->batch_flags, (size_t)count * sizeof(uint32_t));
            if (e == cudaSuccess) e = cudaMallocHost(&cuda->batch_flags_host, (size_t)count * sizeof(uint32_t));
            if (e != cudaSuccess) return fjb::cuda_status(e, error, "batch flag slots");
            cuda->batch_slots = (size_t)count;
        }
        if (cuda->batch_boost.size() < (size_t)count) cuda->batch_boost.resize((size_t)count, nullptr);
        for (int32_t i = 0; i < count && e == cudaSuccess; ++i)
            if (prepared[i]->optics.flags & FJ_OPTICS_HIGHLIGHT_BOOST) e = ensure_boost(cuda->batch_boost[i]);
        if (e != cudaSuccess) return fjb::cuda_status(e, error, "highlight boost state");

        auto outcomes_from = [&](std::vector<FrameWork>& works) {
            FjStatus first = fjb::ok_status();
            for (int32_t i = 0; i < count; ++i) {
                outcomes[i] = frame_outcome(works[i], cuda->batch_flags_host[i], s, error);
                if (first.category == FJ_STATUS_SUCCESS && outcomes[i].status.category != FJ_STATUS_SUCCESS)
                    first = outcomes[i].status;
            }
            return first;
        };
        if (graph && cuda->batch_exec && cuda->batch_token == graph_token && cuda->batch_frames == count) {
            // replay: the frames' work, their flag-word copies and the read-back in one launch
            e = cudaGraphLaunch(cuda->batch_exec, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return fjb::cuda_status(e, error, "batch graph");
            std::vector<FrameWork> works((size_t)count);
            for (int32_t i = 0; i < count; ++i) {
                works[i].boost = (prepared[i]->optics.flags & FJ_OPTICS_HIGHLIGHT_BOOST) != 0;
                works[i].boost_state = cuda->batch_boost[i];
            }
            return outcomes_from(works);
        }
        // every frame in order on one stream, each followed by the copy of its flag word
        // into its slot; one read-back of all slots at the end
        const FjAbortCallback none{nullptr, nullptr};
        auto enqueue_all = [&](std::vector<FrameWork>& works, bool record) -> FjStatus {
            for (int32_t i = 0; i < count; ++i) {
                FjStatus st = frame_enqueue(cuda, &frames[i], submissions ? &submissions[i] : nullptr, prepared[i],
                                            none, s, cuda->batch_boost[i], works[i], error);
                if (st.category != FJ_STATUS_SUCCESS) {
                    if (record) outcomes[i].status = st;
                    return st;
                }
                const cudaError_t ce = cudaMemcpyAsync(cuda->batch_flags + i, works[i].recipe->r.flags, sizeof(uint32_t),
                                                       cudaMemcpyDeviceToDevice, s);
                if (ce != cudaSuccess) return fjb::cuda_status(ce, error, "batch flag copy");
            }
            const cudaError_t ce = cudaMemcpyAsync(cuda->batch_flags_host, cuda->batch_flags,
                                                   (size_t)count * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
            if (ce != cudaSuccess) return fjb::cuda_status(ce, error, "batch flag read-back");
            return fjb::ok_status();
        };
        // per-stage timing covers single frames only
        struct Restore {
            FjCuda* c;
            bool t;
            ~Restore() {
                c->timing = t;
                c->capturing = false;
            }
        } restore{cuda, cuda->timing};
        cuda->timing = false;
        std::vector<FrameWork> works((size_t)count);
        FjStatus st = enqueue_all(works, true);
        const cudaError_t se = cudaStreamSynchronize(s);
        if (st.category != FJ_STATUS_SUCCESS) return st;
        if (se != cudaSuccess) return fjb::cuda_status(se, error, "batch");
        const FjStatus result = outcomes_from(works);
        if (graph) {
            // capture the same enqueue (the owner's caches are warm now) for later calls
            // with this token
            batch_graph_release(cuda);
            cuda->capturing = true;
            std::vector<FrameWork> again((size_t)count);
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
            FjStatus cst = e == cudaSuccess ? enqueue_all(again, false) : fjb::cuda_status(e, nullptr, "capture");
            const cudaError_t ee = e == cudaSuccess ? cudaStreamEndCapture(s, &g) : e;
            cuda->capturing = false;
            if (cst.category == FJ_STATUS_SUCCESS && ee == cudaSuccess && g) {
                cudaGraphExec_t exec = nullptr;
                if (cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) {
                    cuda->batch_exec = exec;
                    cuda->batch_token = graph_token;
                    cuda->batch_frames = count;
                }
            }
            if (g) cudaGraphDestroy(g);
            cudaGetLastError(); // a capture the runtime refused leaves the eager results standing
            if (result.category == FJ_STATUS_SUCCESS)
                fjb::write_error(error, cuda->batch_exec ? "" : "batch graph not captured");
        }
        return result;
    } catch (...) {
        return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_render_batch");
    }
}

FjStatus fjb_owner_set_autotune(FjCuda* cuda, int32_t enable, FjErrorBuffer* error) {
    if (!cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null owner");
    std::lock_guard<std::mutex> lock(cuda->gate);
    cuda->autotune = enable != 0;
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fjb_owner_diffusion_form(FjCuda* cuda, int32_t width, int32_t height, int32_t radius_px, int32_t* form,
                                  FjErrorBuffer* error) {
    if (!cuda || !form) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    std::lock_guard<std::mutex> lock(cuda->gate);
    const auto it = cuda->diffusion_form.find(diffusion_form_key(width, height, radius_px));
    *form = it == cuda->diffusion_form.end() ? -1 : it->second;
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fj_cuda_retire_instance(FjCuda* cuda, uint64_t instance_token, FjErrorBuffer* error) {
    (void)instance_token;
    if (!cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null owner");
    std::lock_guard<std::mutex> lock(cuda->gate);
    if (cuda->closed) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fj_cuda_shutdown(FjCuda* cuda, FjErrorBuffer* error) {
    if (!cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null owner");
    std::lock_guard<std::mutex> lock(cuda->gate);
    if (!cuda->closed) {
        release_all(cuda);
        cuda->closed = true;
    }
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fjb_owner_set_print_form(FjCuda* cuda, int32_t form, FjErrorBuffer* error) {
    if (!cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null owner");
    if (form != FJB_PRINT_FP32 && form != FJB_PRINT_TENSOR && form != FJB_PRINT_TENSOR_SPLIT)
        return fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "unknown print form");
    std::lock_guard<std::mutex> lock(cuda->gate);
    if (cuda->closed) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
    cuda->print_form = form;
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fjb_owner_stage_timing(FjCuda* cuda, int32_t enable, FjErrorBuffer* error) {
    if (!cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null owner");
    std::lock_guard<std::mutex> lock(cuda->gate);
    if (cuda->closed) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
    if (enable && !cuda->timing_events) {
        for (cudaEvent_t& e : cuda->stage_ev) {
            cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) {
                stage_events_release(cuda);
                return fjb::cuda_status(err, error, "stage timing events");
            }
        }
        cuda->timing_events = true;
    }
    cuda->timing = enable != 0;
    for (int s = 0; s < FJB_STAGE_COUNT; ++s) {
        cuda->stage_ms[s] = 0.0;
        cuda->stage_frames[s] = 0;
        cuda->stage_open[s] = false;
    }
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fjb_owner_stage_times(FjCuda* cuda, FjbStageTimes* out, FjErrorBuffer* error) {
    if (!cuda || !out) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
    std::lock_guard<std::mutex> lock(cuda->gate);
    for (int s = 0; s < FJB_STAGE_COUNT; ++s) {
        out->total_ms[s] = cuda->stage_ms[s];
        out->frames[s] = cuda->stage_frames[s];
    }
    fjb::write_error(error, "");
    return fjb::ok_status();
}

FjStatus fj_cuda_destroy(FjCuda* cuda, FjErrorBuffer* error) {
    if (!cuda) return fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null owner");
    {
        std::lock_guard<std::mutex> lock(cuda->gate);
        release_all(cuda);
        cuda->closed = true;
    }
    FjCuda* expected = cuda;
    g_live_owner.compare_exchange_strong(expected, nullptr);
    delete cuda;
    fjb::write_error(error, "");
    return fjb::ok_status();
}

} // extern "C"
