// ref_fft_shim.cu -- TEST INFRASTRUCTURE: drives the reference's own cuFFT camera
// diffusion (src/Cuda/Diffusion/JuicerCudaDiffusion.cu: build_spectrum_package,
// launch_stage) the way its executor and resource code do
// (src/Cuda/JuicerCudaExecutor.cpp:1909-1935, src/Cuda/Diffusion/JuicerCudaDiffusionResources.cpp:
// 700-800 and 900-960): the tile extent from the reference's execution descriptor
// (src/DiffusionExecution.cpp:571), an R2C and a C2R plan over that extent with one
// shared work area, the three channel spectra built by the reference, then the stage
// launch over the frame. Built with the reference's sources into
// oracle/_ref/libjuicer_ref_fft.so by oracle/build_ref.py; only the GPU tests load it,
// to compare this library's diffusion with the reference's in output and in time.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <string>

#include "Cuda/Diffusion/JuicerCudaDiffusion.h"
#include "DiffusionExecution.h"
#include "juicer_diffusion_api.h"

// The reference's host exports the diffusion-component preparation that its
// host-behaviour code imports (native/juicer_diffusion_api.h:63). This harness hands the
// components to the stage directly and never prepares them, so the import is answered
// by a stand-in that refuses.
extern "C" FjStatus fj_diffusion_components_prepare(const FjDiffusionSample*, FjDiffusionComponents*,
                                                    FjDiffusionFailure*, FjErrorBuffer*) {
    FjStatus st{};
    st.category = FJ_STATUS_INTERNAL_FAILURE;
    return st;
}

namespace {

struct Buffers {
    float* transform = nullptr;
    void* spectra[3] = {nullptr, nullptr, nullptr};
    void* work = nullptr;
    float* planes[4] = {nullptr, nullptr, nullptr, nullptr};
    cufftHandle r2c = 0, c2r = 0;
    cudaStream_t stream = nullptr;
    ~Buffers() {
        if (stream) cudaStreamDestroy(stream);
        if (transform) cudaFree(transform);
        for (void* p : spectra)
            if (p) cudaFree(p);
        if (work) cudaFree(work);
        for (float* p : planes)
            if (p) cudaFree(p);
        if (r2c) cufftDestroy(r2c);
        if (c2r) cufftDestroy(c2r);
    }
};

} // namespace

extern "C" {

// Camera diffusion of three device planes (R, G, B; width x height, dense) by the
// reference's cuFFT path: dst = (1 - fraction) src + fraction (PSF * src), the PSF from
// the nine components (lambda in pixels, per-channel weights). The first launch fills
// dst; then `iterations` more launches are timed with CUDA events and their mean is
// written to ms_out. Returns 0, or a negative code naming the step that failed.
int ref_fft_diffusion(const double* lambda_px, const double* w_red, const double* w_green, const double* w_blue,
                      int radius, double fraction, const float* src_r, const float* src_g, const float* src_b,
                      float* dst_r, float* dst_g, float* dst_b, int width, int height, int iterations, float* ms_out) {
    using namespace Spektrafilm;
    namespace D = JuicerCuda::Diffusion;
    DiffusionFrameSetDescriptor fs{};
    fs.fullFrame = {0, 0, width, height};
    DiffusionStageFrameDescriptor cam{};
    cam.stage = DiffusionLinearStage::CameraFilmLinear;
    cam.scatterFraction = fraction;
    cam.sample.radiusPixels = radius;
    cam.sample.hash = 1;
    cam.hash = 1;
    fs.camera = cam;
    fs.hash = 1;
    DiffusionExecutionDescriptor desc{};
    std::string why;
    if (!build_diffusion_execution_descriptor(fs, 1, (std::uint64_t)64 << 30, desc, why)) return -1;
    const PlanLayout& L = desc.layout;
    Buffers b;
    if (cufftCreate(&b.r2c) != CUFFT_SUCCESS || cufftCreate(&b.c2r) != CUFFT_SUCCESS) return -2;
    cufftSetAutoAllocation(b.r2c, 0);
    cufftSetAutoAllocation(b.c2r, 0);
    int dims[2] = {L.height, L.width};
    int rin[2] = {L.height, L.physicalRealRowFloats}, rout[2] = {L.height, L.complexWidth};
    size_t w1 = 0, w2 = 0;
    if (cufftMakePlanMany(b.r2c, 2, dims, rin, 1, L.realDistance, rout, 1, L.complexDistance, CUFFT_R2C, 1, &w1) !=
            CUFFT_SUCCESS ||
        cufftMakePlanMany(b.c2r, 2, dims, rout, 1, L.complexDistance, rin, 1, L.realDistance, CUFFT_C2R, 1, &w2) !=
            CUFFT_SUCCESS)
        return -3;
    const size_t work = std::max(w1, w2);
    if (work && cudaMalloc(&b.work, work) != cudaSuccess) return -4;
    if (work && (cufftSetWorkArea(b.r2c, b.work) != CUFFT_SUCCESS || cufftSetWorkArea(b.c2r, b.work) != CUFFT_SUCCESS))
        return -4;
    if (cudaMalloc(&b.transform, L.transformBytes) != cudaSuccess) return -5;
    for (void*& p : b.spectra)
        if (cudaMalloc(&p, L.transformBytes) != cudaSuccess) return -5;
    const size_t plane = (size_t)width * height * sizeof(float);
    for (float*& p : b.planes)
        if (cudaMalloc(&p, plane) != cudaSuccess) return -6;
    // the reference's launchers require a real stream (a blocking one, ordered after the
    // plain copies below)
    if (cudaStreamCreate(&b.stream) != cudaSuccess) return -6;
    cudaStream_t stream = b.stream;
    if (cufftSetStream(b.r2c, stream) != CUFFT_SUCCESS || cufftSetStream(b.c2r, stream) != CUFFT_SUCCESS) return -3;
    D::SpectrumBuildRequest req{};
    req.layout = L;
    for (int i = 0; i < 9; ++i) {
        req.components.lambdaPixels[i] = lambda_px[i];
        req.components.redWeights[i] = w_red[i];
        req.components.greenWeights[i] = w_green[i];
        req.components.blueWeights[i] = w_blue[i];
    }
    req.radiusPixels = radius;
    req.transformBuffer = b.transform;
    req.normalizationScratch = reinterpret_cast<double*>(b.spectra[0]);
    req.normalizationScratchBytes = (size_t)L.transformBytes;
    req.r2cPlan = b.r2c;
    req.destination = {reinterpret_cast<cufftComplex*>(b.spectra[0]), reinterpret_cast<cufftComplex*>(b.spectra[1]),
                       reinterpret_cast<cufftComplex*>(b.spectra[2])};
    req.stream = stream;
    if (!D::build_spectrum_package(req).ok()) return -7;
    auto launch = [&](D::StagePlaneSet& set) {
        D::StageLaunchRequest lr{};
        lr.layout = L;
        lr.geometry = desc.stages[0];
        lr.fullFrame = fs.fullFrame;
        lr.spectra = req.destination;
        lr.execution = {b.transform, b.r2c, b.c2r};
        lr.planes = &set;
        lr.stream = stream;
        return D::launch_stage(lr).ok();
    };
    const float* srcs[3] = {src_r, src_g, src_b};
    float* dsts[3] = {dst_r, dst_g, dst_b};
    for (int c = 0; c < 3; ++c) cudaMemcpy(b.planes[c], srcs[c], plane, cudaMemcpyDeviceToDevice);
    D::StagePlaneSet set{b.planes[0], b.planes[1], b.planes[2], b.planes[3], (size_t)width};
    if (!launch(set)) return -8;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return -8;
    // the stage rotates the plane pointers: the set names the outputs afterwards
    const float* outs[3] = {set.redSensitive, set.greenSensitive, set.blueSensitive};
    for (int c = 0; c < 3; ++c) cudaMemcpy(dsts[c], outs[c], plane, cudaMemcpyDeviceToDevice);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream);
    for (int i = 0; i < iterations; ++i)
        if (!launch(set)) return -9;
    cudaEventRecord(e1, stream);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_out) *ms_out = iterations > 0 ? ms / (float)iterations : 0.0f;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -10;
}

} // extern "C"
