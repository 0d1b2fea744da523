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

#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "../../include/juicer_cuda_api.h"
#include "fjb_internal.h"
#include "fjb_recipe.h"
#include "fjb_schedule.h"

struct FjCuda {
    std::mutex gate;
    bool closed = false;
    int device = -1;
    std::map<uint64_t, fjb::Recipe*> recipes; // keyed by recipe_hash (non-zero only)
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

void release_all(FjCuda* cuda) {
    for (auto& kv : cuda->recipes) {
        kv.second->release();
        delete kv.second;
    }
    cuda->recipes.clear();
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
        (void)submission;
        std::lock_guard<std::mutex> lock(cuda->gate);
        if (cuda->closed) {
            out.status = fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "owner is shut down");
            return out;
        }
        int dev = 0;
        cudaGetDevice(&dev);
        if (context->device_id != dev) {
            out.status = fjb::fail_status(FJ_STATUS_CONTEXT_LOSS, error, "current device differs from the inspected one");
            return out;
        }
        if (!image_ok(frame->source) || !image_ok(frame->destination) ||
            frame->source.components != frame->destination.components ||
            !rect_inside(frame->render_window, frame->source.bounds) ||
            !rect_inside(frame->render_window, frame->destination.bounds)) {
            out.status = fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "frame images or render window rejected");
            return out;
        }
        if (aborted(abort_callback)) {
            out.status = fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
            return out;
        }
        const bool hostStream = (frame->flags & FJ_FRAME_STREAM_PRESENT) != 0;
        cudaStream_t stream = hostStream ? reinterpret_cast<cudaStream_t>(frame->stream) : nullptr;

        const uint32_t spatialOptics = prepared->optics.flags;
        const bool grain = (prepared->grain.flags & FJ_GRAIN_ACTIVE) != 0;
        const bool spatialDir = prepared->spatial_dir.component_count > 0;
        if (spatialOptics != 0 || grain || spatialDir) {
            out.status = fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error,
                                          "spatial stages are not enabled in this fj_cuda_render build");
            return out;
        }
        if (prepared->film_exposure.flags & FJ_FILM_AUTO_EXPOSURE) {
            out.status = fjb::fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error,
                                          "auto exposure is not enabled in this fj_cuda_render build");
            return out;
        }

        // ---- recipe tables (cached by recipe_hash) ----
        fjb::Recipe* recipe = nullptr;
        fjb::Recipe transient;
        const uint64_t key = prepared->recipe_hash;
        if (key != 0) {
            auto it = cuda->recipes.find(key);
            if (it != cuda->recipes.end()) recipe = it->second;
        }
        if (!recipe) {
            auto* fresh = key != 0 ? new fjb::Recipe() : &transient;
            std::string why;
            FjStatus st{};
            if (!fjb::create_recipe(*prepared, stream, *fresh, why, st)) {
                if (fresh != &transient) delete fresh;
                fjb::write_error(error, why);
                out.status = st;
                return out;
            }
            if (key != 0) cuda->recipes[key] = fresh;
            recipe = fresh;
        }
        if (aborted(abort_callback)) {
            if (recipe == &transient) transient.release();
            out.status = fjb::fail_status(FJ_STATUS_CANCELLED, error, "abort requested");
            return out;
        }

        const FjRect& w = frame->render_window;
        fjb::PixelParams p = recipe->params;
        p.src = pixel_address(frame->source, w.x1, w.y1);
        p.dst = const_cast<char*>(pixel_address(frame->destination, w.x1, w.y1));
        p.src_row_bytes = frame->source.row_bytes;
        p.dst_row_bytes = frame->destination.row_bytes;
        p.width = w.x2 - w.x1;
        p.height = w.y2 - w.y1;
        p.components = (int)frame->source.components;
        cudaError_t e = cudaMemsetAsync(recipe->flags, 0, sizeof(unsigned), stream);
        if (e == cudaSuccess) e = fjb::launch_pixel_chain(p, fjb::PixelStage::SourceToOutput, stream);
        unsigned flags = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&flags, recipe->flags, sizeof(unsigned), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (recipe == &transient) transient.release();
        if (e != cudaSuccess) {
            out.status = fjb::cuda_status(e, error, "render");
            return out;
        }
        if (flags & (1u << 8)) out.flags |= FJ_RENDER_DEFERRED_DIR_ERROR;
        out.status = fjb::ok_status();
        fjb::write_error(error, (flags & 1u) ? "scanner stage reported non-finite pixels" : "");
        return out;
    } catch (...) {
        out.status = fjb::fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fj_cuda_render");
        return out;
    }
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
