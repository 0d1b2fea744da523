// fjb_api_highlight_boost.cpp -- extern "C" entries of the highlight reconstruction
// stage (reference src/Cuda/Film/JuicerCudaHighlightBoost.cu:207-258
// launch_highlight_boost, src/ProcessRoot.cpp:4063-4096 check_highlight_boost).
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/juicer_b200.h"
#include "fjb_highlight_boost.h"
#include "fjb_schedule.h"

using fjb::cuda_status;
using fjb::fail_status;
using fjb::ok_status;
using fjb::write_error;

extern "C" {

size_t fjb_highlight_boost_state_bytes(void) { return sizeof(fjb::BoostState); }

FjStatus fjb_highlight_boost(const FjHighlightBoost* d, float* carrier_b, float* carrier_g, float* carrier_r,
                             ptrdiff_t carrier_stride, int32_t width, int32_t height, void* state, void* stream,
                             FjErrorBuffer* error) {
    try {
        if (!d || !carrier_b || !carrier_g || !carrier_r || !state)
            return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        if (carrier_b == carrier_g || carrier_b == carrier_r || carrier_g == carrier_r || carrier_stride < width ||
            width < 0 || height < 0)
            return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "highlight boost carrier planes");
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        fjb::BoostState* st = static_cast<fjb::BoostState*>(state);
        cudaError_t e = cudaSuccess;
        if (d->recipe_hash == 0 || width == 0 || height == 0) {
            // inactive descriptor: nothing applied (disposition bypass)
            e = cudaMemsetAsync(st, 0, sizeof(fjb::BoostState), s);
        } else {
            const fjb::BoostDescriptor bd{d->protection, d->sharpness, d->peak_gain};
            e = fjb::launch_highlight_boost(bd, carrier_b, carrier_g, carrier_r, carrier_stride, width, height, st, s);
        }
        if (e != cudaSuccess) return cuda_status(e, error, "highlight boost");
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_highlight_boost");
    }
}

FjStatus fjb_highlight_boost_result(const void* state, void* stream, uint32_t* disposition, FjErrorBuffer* error) {
    try {
        if (!state) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        fjb::BoostState host{};
        cudaError_t e = cudaMemcpyAsync(&host, state, sizeof(host), cudaMemcpyDeviceToHost,
                                        reinterpret_cast<cudaStream_t>(stream));
        if (e == cudaSuccess) e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return cuda_status(e, error, "highlight boost result");
        if (disposition) *disposition = host.disposition;
        switch ((int)host.disposition) {
            case fjb::kBoostApplied:
            case fjb::kBoostBypass:
                write_error(error, "");
                return ok_status();
            case fjb::kBoostInvalidCarrier:
                return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "HighlightBoostInvalidCarrier");
            case fjb::kBoostPeakOverflow:
                return fail_status(FJ_STATUS_UNSUPPORTED_INPUT, error, "HighlightBoostPeakOverflow");
        }
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "invalid highlight boost disposition");
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_highlight_boost_result");
    }
}

} // extern "C"
