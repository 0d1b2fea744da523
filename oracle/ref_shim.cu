// ref_shim.cu -- drives the reference's own CUDA render kernels (TEST INFRASTRUCTURE).
//
// Built by oracle/build_ref.py against the read-only reference sources
// (src/Cuda/Scan/JuicerCudaScanPipeline.cu, src/Cuda/Film/JuicerCudaFilmPipeline.cu)
// into oracle/_ref/libjuicer_ref.so. It fills the reference's internal payload
// structs (src/Cuda/JuicerCudaPayloads.h) from an FjPreparedHostData exactly as the
// reference's host packing does (src/Cuda/JuicerCudaFilmPayloads.cpp:28-197,
// src/Cuda/JuicerCudaResources.cpp:3838-3840, :3910-3922, :4186-4254, :4335-4420,
// src/Cuda/JuicerCudaExecutor.cpp:962-1011, :1575-1607), uploads the tables, and
// calls the reference launchers juicer_cuda_negative_pipeline /
// juicer_cuda_print_pipeline / juicer_cuda_direct_focused_capture_density. Only the
// GPU parity tests load it; the product never does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "Cuda/JuicerCudaPayloads.h"
#include "GamutCompression.h"
#include "juicer_cuda_api.h"

extern "C" cudaError_t juicer_cuda_negative_pipeline(const JuicerCuda::PipelineRunParams*, void*);
extern "C" cudaError_t juicer_cuda_print_pipeline(const JuicerCuda::PipelineRunParams*, void*);
extern "C" cudaError_t juicer_cuda_print_focused_capture_density(const JuicerCuda::PrintPipelineRunParams*, float*,
                                                                  float*, float*, void*);

namespace {

struct Arena {
    std::vector<void*> ptrs;
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    const T* put(const T* host, size_t count) {
        void* d = nullptr;
        if (count == 0) return nullptr;
        if (cudaMalloc(&d, count * sizeof(T)) != cudaSuccess) return nullptr;
        cudaMemcpy(d, host, count * sizeof(T), cudaMemcpyHostToDevice);
        ptrs.push_back(d);
        return static_cast<const T*>(d);
    }
    const float* column(const float* src, size_t n, int stride, int col) {
        std::vector<float> v(n);
        for (size_t i = 0; i < n; ++i) v[i] = src[i * stride + col];
        return put(v.data(), n);
    }
};

// Device time of the last reference launcher call (CUDA events around the launcher
// only, after every upload), for the speed comparisons of the GPU tests.
float g_last_ms = 0.0f;

struct LaunchTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    LaunchTimer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaDeviceSynchronize();
        cudaEventRecord(a, nullptr);
    }
    void stop() {
        cudaEventRecord(b, nullptr);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&g_last_ms, a, b);
    }
    ~LaunchTimer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

JuicerCuda::DeviceCurveView curve(const float* x, const float* y, int n) {
    JuicerCuda::DeviceCurveView c{};
    c.x = x;
    c.y = y;
    c.n = n;
    c.domainBegin = 0;
    c.domainEnd = n - 1;
    return c;
}

// Fills a PipelineRunParams the way the reference host does. Returns false on a
// malformed record.
bool pack(const FjPreparedHostData& h, const float* const lut[6], Arena& a, JuicerCuda::PipelineRunParams& p,
          unsigned* d_flags) {
    using namespace JuicerCuda;
    p = PipelineRunParams{};
    const FjFilmExposure& ex = h.film_exposure;
    p.filmRaw.inputColorSpaceIndex = (int)ex.input_color_space;
    p.filmRaw.applyCctfDecoding = (ex.flags & FJ_FILM_DECODE_CCTF) ? 1 : 0;
    p.filmRaw.applyInputChromaticAdapt = (ex.flags & FJ_FILM_ADAPT_INPUT) ? 1 : 0;
    p.filmRaw.rgbToRawMethod = (int)ex.method;
    p.filmRaw.mallettGreenMidgrayScale = ex.mallett_green_midgray_scale;
    std::memcpy(p.filmRaw.inputRGBToXYZ, ex.input_rgb_to_xyz, 36);
    std::memcpy(p.filmRaw.inputXYZAdapt, ex.input_xyz_adapt, 36);
    std::memcpy(p.filmRaw.xyzToLinearSrgb, ex.xyz_to_linear_srgb, 36);
    p.filmExpose.manualExposureScale = std::exp2(ex.manual_exposure_ev);
    p.filmExpose.routeCorrectionScale = ex.route_correction_scale;
    auto& rc = p.filmExpose.reconstruction;
    rc.sensB = curve(nullptr, a.column(ex.sensitivity_rgb.data, 81, 3, 2), 81);
    rc.sensG = curve(nullptr, a.column(ex.sensitivity_rgb.data, 81, 3, 1), 81);
    rc.sensR = curve(nullptr, a.column(ex.sensitivity_rgb.data, 81, 3, 0), 81);
    if (ex.method == FJ_RAW_MALLETT_2019) {
        rc.tablesIllum = a.put(ex.mallett_illuminant.data, 81);
        rc.tablesK = 81;
        rc.mallettBasis = a.put(ex.mallett_basis.data, 243);
        rc.mallettBasisK = 81;
    } else {
        rc.filmTcLut = a.put(ex.tc_lut_rgba.data, ex.tc_lut_rgba.count);
        rc.filmTcLutExtent = kFilmTcLutExtent;
    }
    const FjFilmDevelopment& dv = h.film_development;
    const int n = (int)dv.log_exposure.count;
    const float* dx = a.put(dv.log_exposure.data, n);
    const float* yB = a.column(dv.density_rgb.data, n, 3, 2);
    const float* yG = a.column(dv.density_rgb.data, n, 3, 1);
    const float* yR = a.column(dv.density_rgb.data, n, 3, 0);
    p.filmDevelop.gammaFactorB = dv.gamma_rgb[2];
    p.filmDevelop.gammaFactorG = dv.gamma_rgb[1];
    p.filmDevelop.gammaFactorR = dv.gamma_rgb[0];
    p.filmDevelop.densB = curve(dx, yB, n);
    p.filmDevelop.densG = curve(dx, yG, n);
    p.filmDevelop.densR = curve(dx, yR, n);
    const FjDirCouplers& dir = h.dir_couplers;
    if (dir.mode != FJ_DIR_INACTIVE) {
        p.filmDevelop.dir.mode = static_cast<DirMode>(dir.mode);
        for (int d = 0; d < 3; ++d) {
            for (int r = 0; r < 3; ++r) p.filmDevelop.dir.M[d * 3 + r] = dir.matrix_rgb[(2 - d) * 3 + (2 - r)];
            p.filmDevelop.dir.dMax[d] = dir.density_max_rgb[2 - d];
            p.filmDevelop.dir.dRef[d] = dir.density_ref_rgb[2 - d];
            p.filmDevelop.dir.donorK[d] = dir.donor_k_rgb[2 - d];
            p.filmDevelop.dir.receiverCRef[d] = dir.receiver_c_ref_rgb[2 - d];
            p.filmDevelop.dir.receiverKr[d] = dir.receiver_kr_rgb[2 - d];
        }
        p.filmDevelop.dirDensB = curve(a.put(dir.compensated_axes_rgb[2].data, n), yB, n);
        p.filmDevelop.dirDensG = curve(a.put(dir.compensated_axes_rgb[1].data, n), yG, n);
        p.filmDevelop.dirDensR = curve(a.put(dir.compensated_axes_rgb[0].data, n), yR, n);
    }
    const bool print = h.route == FJ_ROUTE_NEGATIVE_PRINT || h.route == FJ_ROUTE_POSITIVE_PRINT;
    if (print) {
        const FjPrint& pr = h.print;
        p.printExpose.active = 1;
        auto& nt = p.printExpose.negTables;
        nt.epsC = a.column(pr.film_density_cmy.data, 81, 3, 0);
        nt.epsM = a.column(pr.film_density_cmy.data, 81, 3, 1);
        nt.epsY = a.column(pr.film_density_cmy.data, 81, 3, 2);
        nt.baseDensityMin = a.put(pr.film_base_density.data, 81);
        nt.K = 81;
        nt.hasBaseline = 1;
        nt.invYn = 1.0f;
        p.printExpose.printIllumFiltered = a.put(pr.main_illuminant.data, 81);
        p.printExpose.printIllumK = 81;
        p.printExpose.printSensC = curve(nullptr, a.column(pr.sensitivity_cmy.data, 81, 3, 0), 81);
        p.printExpose.printSensM = curve(nullptr, a.column(pr.sensitivity_cmy.data, 81, 3, 1), 81);
        p.printExpose.printSensY = curve(nullptr, a.column(pr.sensitivity_cmy.data, 81, 3, 2), 81);
        p.printExpose.printExposure = pr.exposure;
        p.printExpose.routeCorrectionScale = h.scanner_correction.exposure_scale;
        const bool pf = (pr.flags & FJ_PRINT_PREFLASH) != 0;
        p.printExpose.printPreflashExposure = pf ? pr.preflash_exposure : 0.0f;
        p.printExpose.printMidgrayFactor = pr.normalizer;
        for (int c = 0; c < 3; ++c) p.printExpose.printPreflashRaw[c] = pf ? pr.preflash_raw_cmy[c] : 0.0f;
        const int np = (int)pr.log_exposure.count;
        const float* px = a.put(pr.log_exposure.data, np);
        p.printDevelop.printDcC = curve(px, a.column(pr.density_cmy.data, np, 3, 0), np);
        p.printDevelop.printDcM = curve(px, a.column(pr.density_cmy.data, np, 3, 1), np);
        p.printDevelop.printDcY = curve(px, a.column(pr.density_cmy.data, np, 3, 2), np);
    }
    auto& sc = p.scanStage;
    const int r = (int)h.scanner_lut.resolution;
    const size_t nodes = (size_t)r * r * r * 3, cells = (size_t)(r - 1) * (r - 1) * (r - 1) * 3;
    sc.scanLutLog2PchipXYZ = a.put(lut[0], nodes);
    sc.scanLutPchipSlopeC = a.put(lut[1], nodes);
    sc.scanLutPchipSlopeM = a.put(lut[2], nodes);
    sc.scanLutPchipSlopeY = a.put(lut[3], nodes);
    sc.scanLutPchipCellMin = a.put(lut[4], cells);
    sc.scanLutPchipCellMax = a.put(lut[5], cells);
    sc.scanLutRes = r;
    sc.densityRange.mediumIsNegative = print ? 0 : 1;
    for (int c = 0; c < 3; ++c) {
        sc.densityRange.min_cmy[c] = print ? h.scanner_bounds.min_cmy[c] : -h.scanner_bounds.min_cmy[c];
        sc.densityRange.inv_max_cmy[c] = h.scanner_bounds.inv_span_cmy[c];
    }
    const FjOutputColor& oc = h.output_color;
    std::memcpy(sc.scanColor.cat02, oc.cat02, 36);
    std::memcpy(sc.scanColor.xyzToRgb, oc.xyz_to_rgb, 36);
    std::memcpy(sc.scanColor.illuminantXYZ, oc.illuminant_xyz, 12);
    if (oc.flags & FJ_COLOR_GAMUT_COMPRESSION) {
        sc.scanColor.outputGamutCmax = a.put(oc.gamut_cmax.data, oc.gamut_cmax.count);
        std::memcpy(sc.scanColor.outputGamutNativeRgbToD65Xyz, oc.native_rgb_to_d65_xyz, 36);
        std::memcpy(sc.scanColor.outputGamutD65XyzToNativeRgb, oc.d65_xyz_to_native_rgb, 36);
        std::memcpy(sc.scanColor.outputGamutOklabXyzToLms, Gamut::kOklabXyzToLms.data(), 36);
        std::memcpy(sc.scanColor.outputGamutOklabLmsToXyz, Gamut::kOklabLmsToXyz.data(), 36);
        std::memcpy(sc.scanColor.outputGamutOklabLmsRootToLab, Gamut::kOklabLmsRootToLab.data(), 36);
        std::memcpy(sc.scanColor.outputGamutOklabLabToLmsRoot, Gamut::kOklabLabToLmsRoot.data(), 36);
        std::memcpy(sc.scanColor.outputGamutLightnessKnee, oc.lightness_knee, 12);
        std::memcpy(sc.scanColor.outputGamutChromaKnee, oc.chroma_knee, 12);
        sc.scanColor.outputGamutActive = 1;
    }
    sc.scanColor.encoding.outputColorSpaceIndex = (int)oc.color_space;
    sc.scanColor.encoding.applyCctfEncoding = (oc.flags & FJ_COLOR_ENCODE_CCTF) ? 1 : 0;
    sc.scanColor.encoding.inputIsOutputSpace = (oc.flags & FJ_COLOR_INPUT_IS_OUTPUT_SPACE) ? 1 : 0;
    sc.scanColor.encoding.cctf.kind = (int)oc.encoding.cctf_kind;
    sc.scanColor.encoding.cctf.gamma = oc.encoding.gamma;
    sc.scanColor.encoding.cctf.a = oc.encoding.a;
    sc.scanColor.encoding.cctf.b = oc.encoding.b;
    sc.scanColor.encoding.cctf.c = oc.encoding.c;
    sc.scanColor.encoding.cctf.d = oc.encoding.d;
    sc.scanColor.encoding.cctf.linearCutoff = oc.encoding.linear_cutoff;
    std::memcpy(sc.scanColor.encoding.dwgToOutput, oc.encoding.dwg_to_output, 36);
    sc.correctionActive = (h.scanner_correction.flags & FJ_CORRECTION_ACTIVE) ? 1 : 0;
    sc.correctionSlope = h.scanner_correction.xyz_slope;
    sc.correctionOffset = h.scanner_correction.xyz_offset;
    sc.scanErrorFlag = reinterpret_cast<int*>(d_flags);
    return true;
}

} // namespace

// Renders with the reference kernels. src/dst are device pointers; lut holds the six
// host arrays of the scanner LUT. Synchronous. Returns a cudaError_t value.
extern "C" int ref_render(const FjPreparedHostData* h, const float* const* lut, const float* src,
                          long src_row_bytes, float* dst, long dst_row_bytes, int width, int height, int comps,
                          unsigned* flags_out) {
    Arena a;
    unsigned* d_flags = nullptr;
    if (cudaMalloc(&d_flags, sizeof(unsigned)) != cudaSuccess) return 2;
    cudaMemset(d_flags, 0, sizeof(unsigned));
    a.ptrs.push_back(d_flags);
    JuicerCuda::PipelineRunParams p;
    if (!pack(*h, lut, a, p, d_flags)) return 1;
    p.src = src;
    p.srcRowBytes = (size_t)src_row_bytes;
    p.dst = dst;
    p.dstRowBytes = (size_t)dst_row_bytes;
    p.width = width;
    p.height = height;
    p.nComponents = comps;
    LaunchTimer timer;
    cudaError_t e = p.printExpose.active ? juicer_cuda_print_pipeline(&p, nullptr)
                                         : juicer_cuda_negative_pipeline(&p, nullptr);
    timer.stop();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    unsigned f = 0;
    cudaMemcpy(&f, d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (flags_out) *flags_out = f;
    return (int)e;
}

// Capture density (C, M, Y planes) with the reference kernel.
extern "C" int ref_capture_density(const FjPreparedHostData* h, const float* const* lut, const float* src,
                                   long src_row_bytes, int width, int height, int comps, float* c, float* m,
                                   float* y) {
    Arena a;
    unsigned* d_flags = nullptr;
    if (cudaMalloc(&d_flags, sizeof(unsigned)) != cudaSuccess) return 2;
    cudaMemset(d_flags, 0, sizeof(unsigned));
    a.ptrs.push_back(d_flags);
    JuicerCuda::PipelineRunParams p;
    if (!pack(*h, lut, a, p, d_flags)) return 1;
    JuicerCuda::PrintPipelineRunParams q{};
    q.src = src;
    q.srcRowBytes = (size_t)src_row_bytes;
    q.dst = c; // unused by the capture kernel but must be non-null for some guards
    q.dstRowBytes = (size_t)src_row_bytes;
    q.width = width;
    q.height = height;
    q.nComponents = comps;
    q.filmExpose = p.filmExpose;
    q.filmDevelop = p.filmDevelop;
    q.printExpose = p.printExpose;
    q.printDevelop = p.printDevelop;
    q.scanStage = p.scanStage;
    q.filmRaw = p.filmRaw;
    LaunchTimer timer;
    cudaError_t e = juicer_cuda_print_focused_capture_density(&q, c, m, y, nullptr);
    timer.stop();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

#include "Cuda/Film/JuicerCudaScatterHalation.h"
#include "ScatterHalation.h"

// Scatter/halation with the reference's own kernels
// (src/Cuda/Film/JuicerCudaScatterHalation.cu:690 launch_scatter_halation). planes are
// device pointers (R, G, B) with `stride` floats per row; modified in place.
extern "C" int ref_scatter_halation(const FjScatterHalation* d, float* r, float* g, float* b, long stride, int width,
                                    int height) {
    ScatterHalationFrameDescriptor desc{};
    desc.recipeHash = d->recipe_hash ? d->recipe_hash : 1;
    desc.scatterAmount = d->scatter_amount;
    desc.bounceCount = d->bounce_count;
    for (int i = 0; i < 5; ++i) desc.bounceWeights[i] = d->bounce_weights[i];
    desc.renormalize = d->renormalize != 0;
    auto conv = [](const FjHalationGaussian& s) {
        ScatterHalationGaussianDescriptor o{};
        o.kind = static_cast<ScatterHalationGaussianKind>(s.kind);
        o.radius = s.radius;
        for (int i = 0; i < 19; ++i) o.firWeights[i] = s.fir_weights[i];
        for (int i = 0; i < 4; ++i) o.yvv[i] = s.yvv[i];
        return o;
    };
    for (int c = 0; c < 3; ++c) {
        const FjHalationChannel& ch = d->channels[c];
        desc.channels[c].core = conv(ch.core);
        for (int i = 0; i < 3; ++i) desc.channels[c].tail[i] = conv(ch.tail[i]);
        for (int i = 0; i < 5; ++i) desc.channels[c].bounce[i] = conv(ch.bounce[i]);
        desc.channels[c].totalStrength = ch.total_strength;
        desc.channels[c].tailWeight = ch.tail_weight;
    }
    float* temp = nullptr;
    float* acc = nullptr;
    const size_t bytes = (size_t)width * height * sizeof(float);
    if (cudaMalloc(&temp, bytes) != cudaSuccess) return 2;
    if (cudaMalloc(&acc, bytes) != cudaSuccess) {
        cudaFree(temp);
        return 2;
    }
    JuicerCuda::ScatterHalationPreparedView view{};
    view.descriptor = &desc;
    view.fullFrameWidth = width;
    view.fullFrameHeight = height;
    view.currentCarrier.redSensitive = r;
    view.currentCarrier.greenSensitive = g;
    view.currentCarrier.blueSensitive = b;
    view.currentCarrier.rowStrideFloats = (size_t)stride;
    view.filterTemp = temp;
    view.weightedAccumulation = acc;
    LaunchTimer timer;
    const JuicerCuda::ScatterHalationLaunchResult res = JuicerCuda::launch_scatter_halation(view, nullptr);
    timer.stop();
    cudaError_t e = res.status;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(temp);
    cudaFree(acc);
    return (int)e;
}

// Spatial DIR with the reference's own kernels (src/Cuda/Film/JuicerCudaFilmPipeline.cu:1479
// juicer_cuda_build_print_spatial_dir). `comps` lists the frame's components in order
// (core first), with boundary weights and FIR taps computed on the host; outputs are
// device planes.
struct RefDirComp {
    int op;
    float weight;
    int radius;
    const float* taps;
    double ff, fb[3];
    const double* h_init;
    int h_len, h_ts;
    double h_term[9];
    const double* v_init;
    int v_len, v_ts;
    double v_term[9];
};

extern "C" cudaError_t juicer_cuda_build_print_spatial_dir(const JuicerCuda::PrintPipelineRunParams*,
                                                          JuicerCuda::SpatialDirBuildRequest);

extern "C" int ref_spatial_dir(const FjPreparedHostData* h, const float* const* lut, const float* src,
                               long src_row_bytes, int width, int height, int comps_n, const RefDirComp* comps,
                               int count, float* fy, float* fm, float* fc, float* lb, float* lg, float* lr) {
    Arena a;
    unsigned* d_flags = nullptr;
    if (cudaMalloc(&d_flags, sizeof(unsigned)) != cudaSuccess) return 2;
    cudaMemset(d_flags, 0, sizeof(unsigned));
    a.ptrs.push_back(d_flags);
    JuicerCuda::PipelineRunParams p;
    if (!pack(*h, lut, a, p, d_flags)) return 1;
    JuicerCuda::PrintPipelineRunParams q{};
    q.src = src;
    q.srcRowBytes = (size_t)src_row_bytes;
    q.dst = fy;
    q.dstRowBytes = (size_t)src_row_bytes;
    q.width = width;
    q.height = height;
    q.nComponents = comps_n;
    q.filmExpose = p.filmExpose;
    q.filmDevelop = p.filmDevelop;
    q.printExpose = p.printExpose;
    q.printDevelop = p.printDevelop;
    q.scanStage = p.scanStage;
    q.filmRaw = p.filmRaw;
    const size_t plane = (size_t)width * height;
    float* work = nullptr;
    if (cudaMalloc(&work, 6 * plane * sizeof(float)) != cudaSuccess) return 2;
    a.ptrs.push_back(work);
    JuicerCuda::SpatialDirBuildRequest req{};
    req.planes.rawCorrectionY = work;
    req.planes.rawCorrectionM = work + plane;
    req.planes.rawCorrectionC = work + 2 * plane;
    req.planes.filterTemp = work + 3 * plane;
    req.planes.filterTempM = work + 4 * plane;
    req.planes.filterTempC = work + 5 * plane;
    req.planes.filteredCorrectionY = fy;
    req.planes.filteredCorrectionM = fm;
    req.planes.filteredCorrectionC = fc;
    req.planes.logRawB = lb;
    req.planes.logRawG = lg;
    req.planes.logRawR = lr;
    JuicerCuda::SpatialDirFilterSpec* specs[4] = {&req.gaussian, &req.tails[0], &req.tails[1], &req.tails[2]};
    for (int k = 0; k < count && k < 4; ++k) {
        const RefDirComp& c = comps[k];
        JuicerCuda::SpatialDirFilterSpec& s = *specs[k];
        s.weight = c.weight;
        s.radius = c.radius;
        s.sigma = 0.0f;
        if (c.op == 1) {
            s.filterOperator = JuicerCuda::SpatialDirFilterOperator::Identity;
        } else if (c.op == 2) {
            s.filterOperator = JuicerCuda::SpatialDirFilterOperator::FirReflect;
            s.kernel = a.put(c.taps, (size_t)(2 * c.radius + 1));
            s.sigma = 1.0f; // eligibility only: FIR requires 0 < sigma < 3
        } else if (c.op == 3) {
            s.filterOperator = JuicerCuda::SpatialDirFilterOperator::YvvReflect;
            s.radius = 0;
            s.sigma = 3.0f; // eligibility only: recursion requires sigma >= 3
            s.iir.feedforward = c.ff;
            for (int i = 0; i < 3; ++i) s.iir.feedback[i] = c.fb[i];
            s.horizontalBoundary.initialWeights = a.put(c.h_init, (size_t)3 * c.h_len);
            s.horizontalBoundary.initialWeightLength = c.h_len;
            s.horizontalBoundary.terminalSize = c.h_ts;
            for (int i = 0; i < 9; ++i) s.horizontalBoundary.terminalMatrix[i] = c.h_term[i];
            s.verticalBoundary.initialWeights = a.put(c.v_init, (size_t)3 * c.v_len);
            s.verticalBoundary.initialWeightLength = c.v_len;
            s.verticalBoundary.terminalSize = c.v_ts;
            for (int i = 0; i < 9; ++i) s.verticalBoundary.terminalMatrix[i] = c.v_term[i];
        }
    }
    LaunchTimer timer;
    cudaError_t e = juicer_cuda_build_print_spatial_dir(&q, req);
    timer.stop();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

extern "C" float ref_last_ms() { return g_last_ms; }

// ---- visual grain: src/Cuda/Scan/JuicerCudaScanPipeline.cu:3141 with the payload
// packing of src/Cuda/JuicerCudaFilmPayloads.cpp:384-495 (stbn offsets :212-240).
extern "C" cudaError_t juicer_cuda_apply_visual_grain(const JuicerCuda::GrainPayload*,
                                                      const JuicerCuda::GrainKernelPayload*, int, int, float*, float*,
                                                      float*, float*, float*, float*, float*, float*, void*);

namespace {

uint64_t fnv_pair(uint64_t a, uint64_t b) {
    uint64_t h = 0xcbf29ce484222325ULL, v[2] = {a, b};
    for (int k = 0; k < 2; ++k)
        for (int i = 0; i < 8; ++i) {
            h ^= (v[k] >> (8 * i)) & 0xFFu;
            h *= 0x100000001b3ULL;
        }
    return h;
}

// Host Gaussian taps as the reference's host preparation callback produces them
// (rust/film-juicer-core/src/optics/gaussian.rs:16-52).
std::vector<float> host_taps(int radius, float sigma) {
    std::vector<float> w((size_t)(2 * radius + 1));
    const double s = (double)sigma, s2 = s * s * 2.0;
    double sum = 0.0;
    for (int i = -radius; i <= radius; ++i) {
        const double v = std::exp(-((double)i * (double)i) / s2);
        w[(size_t)(i + radius)] = (float)v;
        sum += v;
    }
    const double rec = sum != 0.0 ? 1.0 / sum : 0.0;
    for (float& v : w) v = (float)((double)v * rec);
    return w;
}

} // namespace

// Density planes (device, width x height, contiguous) in place. base_cmy: capture
// density curve values (host, n each); layers: 9 host curves [layer][CMY].
extern "C" int ref_visual_grain(const FjVisualGrain* g, const FjStaticNoise* noise, const float* const* base_cmy,
                                const float* const* layers, int n, int positive, float* dc, float* dm, float* dy,
                                int width, int height) {
    Arena a;
    JuicerCuda::GrainPayload p{};
    JuicerCuda::GrainKernelPayload k{};
    const bool sub = (g->flags & FJ_GRAIN_SUBLAYERS) != 0;
    p.active = (g->flags & FJ_GRAIN_ACTIVE) ? 1 : 0;
    p.sublayersActive = sub ? 1 : 0;
    p.positiveFilm = positive;
    p.nSubLayers = (int)g->sublayer_count;
    p.originX = g->render_extent.x;
    p.originY = g->render_extent.y;
    p.seedBase = g->seed_base;
    p.seedBaseNext = g->seed_base_next;
    if (noise) {
        p.stbn = a.put(noise->stbn.data, noise->stbn.count);
        p.stbnWidth = noise->stbn_width;
        p.stbnHeight = noise->stbn_height;
        p.stbnFrames = noise->stbn_frames;
        p.wangTiles = a.put(noise->wang_tiles.data, noise->wang_tiles.count);
        p.wangLut = a.put(noise->wang_lut.data, noise->wang_lut.count);
        p.wangWidth = noise->wang_width;
        p.wangHeight = noise->wang_height;
        p.wangCount = (int)noise->wang_tile_count;
        p.wangColors = noise->wang_colors;
    }
    p.stbnOffsetX = p.stbnWidth > 0 ? (int)(fnv_pair(g->session_seed, 0xA5u) % (uint64_t)p.stbnWidth) : 0;
    p.stbnOffsetY = p.stbnHeight > 0 ? (int)(fnv_pair(g->session_seed, 0x5Au) % (uint64_t)p.stbnHeight) : 0;
    if (p.stbnFrames > 0) {
        const int64_t ph = (int64_t)(g->session_seed % (uint64_t)p.stbnFrames);
        int f = (int)((g->frame0 + ph) % p.stbnFrames);
        p.stbnFrame = f < 0 ? f + p.stbnFrames : f;
    }
    p.frameIndex = g->frame0;
    p.timeAlpha = g->frame_alpha;
    p.stbnSessionSeed = g->session_seed;
    p.clipToken = g->clip_token;
    p.wangCellMm = g->wang_cell_mm;
    p.breathingPeriodFrames = g->breathing_period_frames;
    p.breathingAmplitude = g->breathing_amplitude;
    p.breathingCellUmSmall = g->breathing_cell_um_small;
    p.breathingCellUmLarge = g->breathing_cell_um_large;
    p.breathingMix = g->breathing_mix;
    p.breathingDriftUmPerFrame = g->breathing_drift_um_per_frame;
    p.debugView = (int)g->debug_view;
    p.pixelSizeUm = g->pixel_size_um;
    p.pitchPx = g->pitch_px;
    p.microStructure[0] = g->micro_structure[0];
    p.microStructure[1] = g->micro_structure[1];
    p.clumpTemporalMix = g->clump_temporal_mix;
    p.clumpMorphPeriodFrames = g->clump_morph_period_frames;
    p.sizeMixWeightFine = g->size_mix_weights[0];
    p.sizeMixWeightMid = g->size_mix_weights[1];
    p.sizeMixWeight = g->size_mix_weights[2];
    p.sizeMixScale = g->size_mix_scale;
    p.sizeMixGain = g->size_mix_gain;
    p.amplitude = g->amplitude;
    p.chromaMix = g->chroma_mix;
    p.chromaSharedWeight = g->chroma_shared_weight;
    p.chromaIndWeight = g->chroma_independent_weight;
    p.debugScale = g->debug_scale;
    for (int c = 0; c < 3; ++c) {
        p.densityMin[c] = g->particle_density_min_cmy[c];
        p.uniformity[c] = g->uniformity_cmy[c];
        p.densityMax[c] = g->density_max_cmy[c];
        p.nParticles[c] = g->n_particles_cmy[c];
        p.odParticle[c] = g->od_particle_cmy[c];
        if (sub) {
            const float* y = a.put(base_cmy[c], (size_t)n);
            p.densityCurveCmy[c] = curve(y, y, n);
            p.densityLayerAxisFinite[c] = (g->flags & (FJ_GRAIN_AXIS_FINITE_C << c)) ? 1 : 0;
            for (int b = 0; b < 16; ++b) p.densityLayerAxisBlockPrefixMax[c][b] = g->layer_axis_block_prefix_max[c][b];
        }
    }
    // identical Gaussians (same descriptor hash) share one prepared kernel, as the
    // reference's preparation dedupes them (src/ProcessRoot.cpp:3441-3490)
    std::vector<std::pair<uint64_t, const float*>> prepared;
    auto prep = [&](const FjGrainGaussian& gg) -> const float* {
        if (gg.radius <= 0) return nullptr;
        for (auto& e : prepared)
            if (e.first == gg.hash) return e.second;
        const std::vector<float> w = host_taps(gg.radius, gg.sigma_px);
        const float* d = a.put(w.data(), w.size());
        prepared.push_back({gg.hash, d});
        return d;
    };
    k.blurKernel = prep(g->correlation[0]);
    k.blurRadius = g->correlation[0].radius;
    k.blurKernelMid = prep(g->correlation[1]);
    k.blurRadiusMid = g->correlation[1].radius;
    k.blurKernelCoarse = prep(g->correlation[2]);
    k.blurRadiusCoarse = g->correlation[2].radius;
    for (int l = 0; l < 3; ++l)
        for (int c = 0; c < 3; ++c) {
            p.densityMinLayers[l][c] = g->density_min_layers[l][c];
            p.densityMaxLayers[l][c] = g->density_max_layers[l][c];
            p.nParticlesLayers[l][c] = g->n_particles_layers[l][c];
            p.odParticleLayers[l][c] = g->od_particle_layers[l][c];
            p.densityCurvesLayers[l][c] = sub ? a.put(layers[l * 3 + c], (size_t)n) : nullptr;
            k.dyeKernel[l][c] = sub ? prep(g->dye_cloud[l][c]) : nullptr;
            k.dyeRadius[l][c] = sub ? g->dye_cloud[l][c].radius : 0;
        }
    void* uniforms = nullptr;
    if (cudaMalloc(&uniforms, sizeof(JuicerCuda::GrainFrameUniforms)) != cudaSuccess) return 2;
    a.ptrs.push_back(uniforms);
    p.frameUniforms = static_cast<JuicerCuda::GrainFrameUniforms*>(uniforms);
    float* work = nullptr;
    const size_t plane = (size_t)width * (size_t)height;
    if (cudaMalloc(&work, 5 * plane * sizeof(float)) != cudaSuccess) return 2;
    a.ptrs.push_back(work);
    LaunchTimer timer;
    cudaError_t e = juicer_cuda_apply_visual_grain(&p, &k, width, height, dc, dm, dy, work, work + plane,
                                                   work + 2 * plane, work + 3 * plane, work + 4 * plane, nullptr);
    timer.stop();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

// ---- scanner post effects with the reference's kernels ----
extern "C" cudaError_t juicer_cuda_print_focused_scan_linear_density_rgb(
    const JuicerCuda::PrintPipelineRunParams*, const float*, const float*, const float*, float*, float*, float*,
    float*, float*, int, int, std::uint64_t, float, float, const float*, int, void*);
extern "C" cudaError_t juicer_cuda_print_focused_continue_from_capture_density(
    const JuicerCuda::PrintPipelineRunParams*, float*, float*, float*, const float*, void*);
extern "C" cudaError_t juicer_cuda_print_focused_scanner_post_output(
    const JuicerCuda::PrintPipelineRunParams*, float*, float*, float*, float*, const float*, int, const float*, int,
    float, const JuicerCuda::FilmDefectsPayload*, const JuicerCuda::GateWeavePayload*, const float*, int, int, void*);

namespace {
// rust/film-juicer-core/src/optics/gaussian.rs:18-59 (the host callback's kernel)
std::vector<float> ref_gaussian(int radius, float sigma_px) {
    std::vector<float> w;
    const double sigma = (double)sigma_px, s2 = sigma * sigma * 2.0;
    double sum = 0.0;
    for (int i = -radius; i <= radius; ++i) {
        const double v = std::exp(-((double)i * (double)i) / s2);
        w.push_back((float)v);
        sum += v;
    }
    const double rec = sum != 0.0 ? 1.0 / sum : 0.0;
    for (float& v : w) v = (float)((double)v * rec);
    return w;
}
} // namespace

// Density planes (device) -> print -> scan to linear RGB with glare -> lens blur ->
// unsharp -> encoded dst (device), through the reference's launchers
// (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2982, :3106), scheduled as
// src/Cuda/JuicerCudaExecutor.cpp:2384-2500 does for the materialized-density route.
extern "C" int ref_scanner_post(const FjPreparedHostData* h, const float* const* lut, const FjScannerPostEffects* post,
                                unsigned long long seed, int origin_x, int origin_y, const float* dc, const float* dm,
                                const float* dy, const float* src, long src_row_bytes, float* dst, long dst_row_bytes,
                                int width, int height, int comps) {
    Arena a;
    unsigned* d_flags = nullptr;
    if (cudaMalloc(&d_flags, sizeof(unsigned)) != cudaSuccess) return 2;
    cudaMemset(d_flags, 0, sizeof(unsigned));
    a.ptrs.push_back(d_flags);
    JuicerCuda::PipelineRunParams p;
    if (!pack(*h, lut, a, p, d_flags)) return 1;
    JuicerCuda::PrintPipelineRunParams q{};
    q.src = src;
    q.srcRowBytes = (size_t)src_row_bytes;
    q.dst = dst;
    q.dstRowBytes = (size_t)dst_row_bytes;
    q.width = width;
    q.height = height;
    q.nComponents = comps;
    q.filmExpose = p.filmExpose;
    q.filmDevelop = p.filmDevelop;
    q.printExpose = p.printExpose;
    q.printDevelop = p.printDevelop;
    q.scanStage = p.scanStage;
    q.filmRaw = p.filmRaw;
    const size_t plane = (size_t)width * (size_t)height;
    float* buf = nullptr;
    if (cudaMalloc(&buf, plane * 8 * sizeof(float)) != cudaSuccess) return 2;
    a.ptrs.push_back(buf);
    float *r = buf, *g = buf + plane, *b = buf + 2 * plane, *tmp = buf + 3 * plane, *blurred = buf + 4 * plane;
    // the materialized-density route scans print densities: develop the print first
    // (src/Cuda/JuicerCudaExecutor.cpp develop_print_capture -> :2908)
    float *pc = buf + 5 * plane, *pm = buf + 6 * plane, *py = buf + 7 * plane;
    cudaMemcpy(pc, dc, plane * sizeof(float), cudaMemcpyDeviceToDevice);
    cudaMemcpy(pm, dm, plane * sizeof(float), cudaMemcpyDeviceToDevice);
    cudaMemcpy(py, dy, plane * sizeof(float), cudaMemcpyDeviceToDevice);
    if (p.printExpose.active) {
        cudaError_t pe = juicer_cuda_print_focused_continue_from_capture_density(&q, pc, pm, py, nullptr, nullptr);
        if (pe != cudaSuccess) return (int)pe;
    }
    dc = pc;
    dm = pm;
    dy = py;
    const bool active = post->hash != 0;
    const float* gk = nullptr;
    const float* lk = nullptr;
    const float* uk = nullptr;
    int gr = 0, lr = 0, ur = 0;
    std::vector<float> gw, lw, uw;
    if (active && (post->flags & FJ_POST_GLARE) && post->glare_blur_sigma_px > 0.0f) {
        gw = ref_gaussian(post->glare_blur_radius, post->glare_blur_sigma_px);
        gk = a.put(gw.data(), gw.size());
        gr = post->glare_blur_radius;
    }
    if (active && post->lens_blur_sigma_px > 0.0f) {
        lw = ref_gaussian(post->lens_blur_radius, post->lens_blur_sigma_px);
        lk = a.put(lw.data(), lw.size());
        lr = post->lens_blur_radius;
    }
    if (active && post->unsharp_sigma_px > 0.0f) {
        uw = ref_gaussian(post->unsharp_radius, post->unsharp_sigma_px);
        uk = a.put(uw.data(), uw.size());
        ur = post->unsharp_radius;
    }
    LaunchTimer timer;
    cudaError_t e = juicer_cuda_print_focused_scan_linear_density_rgb(
        &q, dc, dm, dy, r, g, b, active ? tmp : nullptr, active ? blurred : nullptr, origin_x, origin_y,
        (std::uint64_t)seed, active ? post->glare_percent : 0.0f, active ? post->glare_roughness : 0.0f, gk, gr,
        nullptr);
    if (e == cudaSuccess)
        e = juicer_cuda_print_focused_scanner_post_output(&q, r, g, b, active ? tmp : nullptr, lk, lr, uk, ur,
                                                          active ? post->unsharp_amount : 0.0f, nullptr, nullptr,
                                                          nullptr, 0, 0, nullptr);
    timer.stop();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

// ---- highlight reconstruction with the reference's launcher ----
#include "Cuda/Film/JuicerCudaHighlightBoost.h"

// Carrier planes B, G, R (device, `stride` floats per row) boosted in place by
// JuicerCuda::launch_highlight_boost (src/Cuda/Film/JuicerCudaHighlightBoost.cu:207);
// writes the disposition. Returns a cudaError_t value.
extern "C" int ref_highlight_boost(const FjHighlightBoost* d, float* b, float* g, float* r, long stride, int width,
                                   int height, int* disposition) {
    JuicerCuda::HighlightBoostWorkspace* ws = nullptr;
    if (cudaMalloc(&ws, sizeof(*ws)) != cudaSuccess) return 2;
    cudaMemset(ws, 0, sizeof(*ws));
    JuicerCuda::HighlightBoostDescriptor desc{};
    desc.recipeHash = d->recipe_hash;
    desc.protection = d->protection;
    desc.sharpness = d->sharpness;
    desc.peakGain = d->peak_gain;
    JuicerCuda::CameraFilmLinearExposurePlanes carrier{};
    carrier.blueSensitive = b;
    carrier.greenSensitive = g;
    carrier.redSensitive = r;
    carrier.rowStrideFloats = (size_t)stride;
    LaunchTimer timer;
    const auto res = JuicerCuda::launch_highlight_boost(desc, carrier, width, height, ws, nullptr,
                                                        JuicerCuda::kHighlightBoostMaxBlocks);
    timer.stop();
    cudaError_t e = res.status;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    JuicerCuda::HighlightBoostDisposition disp{};
    if (e == cudaSuccess) e = cudaMemcpy(&disp, &ws->disposition, sizeof(disp), cudaMemcpyDeviceToHost);
    if (disposition) *disposition = (int)disp;
    cudaFree(ws);
    return (int)e;
}

// ---- film and gate defects with the reference's kernels ----
extern "C" cudaError_t juicer_cuda_apply_film_defects(const JuicerCuda::FilmDefectsPayload*, int, int, float*, float*,
                                                      float*, float*, void*);
extern "C" cudaError_t juicer_cuda_build_gate_defect_transmittance_focused(const JuicerCuda::FilmDefectsPayload*,
                                                                            float*, int, int, void*);
extern "C" cudaError_t juicer_cuda_direct_focused_scan_linear_density_rgb(const JuicerCuda::DirectPipelineRunParams*,
                                                                          const float*, const float*, const float*,
                                                                          float*, float*, float*, const float*, void*);
extern "C" cudaError_t juicer_cuda_direct_focused_scanner_post_output(
    const JuicerCuda::DirectPipelineRunParams*, float*, float*, float*, float*, const float*, int, const float*, int,
    float, const JuicerCuda::FilmDefectsPayload*, const JuicerCuda::GateWeavePayload*, const float*, int, int, void*);

namespace {
// src/Cuda/JuicerCudaFilmPayloads.cpp:505-688: the record's families, origins and frame
// fields into the payloads (the dust and scratch records list the same fields in the
// same order as the payload structs).
static_assert(sizeof(JuicerCuda::DefectDustPayload) == sizeof(FjDust), "dust layout");
static_assert(sizeof(JuicerCuda::DefectScratchPayload) == sizeof(FjScratch), "scratch layout");
void pack_effects(const FjFilmEffects& e, JuicerCuda::FilmDefectsPayload& d, JuicerCuda::GateWeavePayload& w) {
    d = {};
    w = {};
    if (!(e.flags & (FJ_EFFECTS_FILM | FJ_EFFECTS_GATE_OUTPUT))) return;
    std::memcpy(&d.filmDust, &e.film_dust, sizeof(FjDust));
    std::memcpy(&d.filmScratch, &e.film_scratch, sizeof(FjScratch));
    std::memcpy(&d.gateDust, &e.gate_dust, sizeof(FjDust));
    std::memcpy(&d.gateScratch, &e.gate_scratch, sizeof(FjScratch));
    for (int i = 0; i < 4; ++i)
        d.origins[i] = {e.origins[i].cell_x, e.origins[i].cell_y, e.origins[i].local_x_mm, e.origins[i].local_y_mm};
    d.sampleStepXMm = e.sample_step_x_mm;
    d.sampleStepYMm = e.sample_step_y_mm;
    d.roiOffsetX = e.roi_offset_x;
    d.roiOffsetY = e.roi_offset_y;
    d.sessionSeed = e.session_seed;
    d.clipToken = e.clip_token;
    w.active = (e.flags & FJ_EFFECTS_WEAVE) ? 1 : 0;
    w.dxPx = e.weave_dx_px;
    w.dyPx = e.weave_dy_px;
    w.cosRot = e.weave_cos_rot;
    w.sinRot = e.weave_sin_rot;
}
} // namespace

// Capture density planes (device, modified in place) -> film defects -> print (print
// route, with the dust) -> scan to linear RGB (direct route: with the dust) -> gate
// mask -> output with weave and gate mask, through the reference's launchers as
// src/Cuda/JuicerCudaExecutor.cpp schedules them (:1674-1690 / :2263-2279 film
// defects, :2788-2790 gate mask, :1700-1800 / :2384-2500 scan and output). `dust`
// (width x height) and `mask` (gate grid) are device buffers the caller may read back.
extern "C" int ref_effects_render(const FjPreparedHostData* h, const float* const* lut, const FjFilmEffects* fx,
                                  float* dc, float* dm, float* dy, const float* src, long src_row_bytes, float* dst,
                                  long dst_row_bytes, int width, int height, int comps, float* dust, float* mask) {
    Arena a;
    unsigned* d_flags = nullptr;
    if (cudaMalloc(&d_flags, sizeof(unsigned)) != cudaSuccess) return 2;
    cudaMemset(d_flags, 0, sizeof(unsigned));
    a.ptrs.push_back(d_flags);
    JuicerCuda::PipelineRunParams p;
    if (!pack(*h, lut, a, p, d_flags)) return 1;
    JuicerCuda::FilmDefectsPayload defects;
    JuicerCuda::GateWeavePayload weave;
    pack_effects(*fx, defects, weave);
    const bool film = (fx->flags & FJ_EFFECTS_FILM) != 0;
    const bool output = (fx->flags & FJ_EFFECTS_GATE_OUTPUT) != 0;
    const bool gate = output && (fx->flags & FJ_EFFECTS_GATE_TRANSMITTANCE) != 0;
    const float* dust_t = film && fx->film_dust.slot_probability > 0.0f ? dust : nullptr;
    const size_t plane = (size_t)width * (size_t)height;
    float* buf = nullptr;
    if (cudaMalloc(&buf, plane * 4 * sizeof(float)) != cudaSuccess) return 2;
    a.ptrs.push_back(buf);
    float *r = buf, *g = buf + plane, *b = buf + 2 * plane, *tmp = buf + 3 * plane;
    cudaError_t e = cudaSuccess;
    if (film) e = juicer_cuda_apply_film_defects(&defects, width, height, dc, dm, dy, dust, nullptr);
    if (e == cudaSuccess && gate)
        e = juicer_cuda_build_gate_defect_transmittance_focused(&defects, mask, fx->gate_width, fx->gate_height,
                                                                nullptr);
    if (e != cudaSuccess) return (int)e;
    if (p.printExpose.active) {
        JuicerCuda::PrintPipelineRunParams q{};
        q.src = src;
        q.srcRowBytes = (size_t)src_row_bytes;
        q.dst = dst;
        q.dstRowBytes = (size_t)dst_row_bytes;
        q.width = width;
        q.height = height;
        q.nComponents = comps;
        q.filmExpose = p.filmExpose;
        q.filmDevelop = p.filmDevelop;
        q.printExpose = p.printExpose;
        q.printDevelop = p.printDevelop;
        q.scanStage = p.scanStage;
        q.filmRaw = p.filmRaw;
        e = juicer_cuda_print_focused_continue_from_capture_density(&q, dc, dm, dy, dust_t, nullptr);
        if (e == cudaSuccess)
            e = juicer_cuda_print_focused_scan_linear_density_rgb(&q, dc, dm, dy, r, g, b, nullptr, nullptr, 0, 0, 0,
                                                                  0.0f, 0.0f, nullptr, 0, nullptr);
        if (e == cudaSuccess)
            e = juicer_cuda_print_focused_scanner_post_output(&q, r, g, b, tmp, nullptr, 0, nullptr, 0, 0.0f,
                                                              output ? &defects : nullptr, output ? &weave : nullptr,
                                                              gate ? mask : nullptr, gate ? fx->gate_width : 0,
                                                              gate ? fx->gate_height : 0, nullptr);
    } else {
        JuicerCuda::DirectPipelineRunParams q{};
        q.src = src;
        q.srcRowBytes = (size_t)src_row_bytes;
        q.dst = dst;
        q.dstRowBytes = (size_t)dst_row_bytes;
        q.width = width;
        q.height = height;
        q.nComponents = comps;
        q.filmExpose = p.filmExpose;
        q.filmDevelop = p.filmDevelop;
        q.scanStage = p.scanStage;
        q.filmRaw = p.filmRaw;
        e = juicer_cuda_direct_focused_scan_linear_density_rgb(&q, dc, dm, dy, r, g, b, dust_t, nullptr);
        if (e == cudaSuccess)
            e = juicer_cuda_direct_focused_scanner_post_output(&q, r, g, b, tmp, nullptr, 0, nullptr, 0, 0.0f,
                                                               output ? &defects : nullptr, output ? &weave : nullptr,
                                                               gate ? mask : nullptr, gate ? fx->gate_width : 0,
                                                               gate ? fx->gate_height : 0, nullptr);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

// The reference's film-defect and gate-mask launchers alone, each timed with CUDA
// events (ref_last_ms after each call): `which` 0 film defects (density planes in
// place, dust plane), 1 gate mask (gate grid).
extern "C" int ref_defects_timed(const FjFilmEffects* fx, int which, int width, int height, float* dc, float* dm,
                                 float* dy, float* out) {
    JuicerCuda::FilmDefectsPayload defects;
    JuicerCuda::GateWeavePayload weave;
    pack_effects(*fx, defects, weave);
    LaunchTimer timer;
    cudaError_t e = which == 0
                        ? juicer_cuda_apply_film_defects(&defects, width, height, dc, dm, dy, out, nullptr)
                        : juicer_cuda_build_gate_defect_transmittance_focused(&defects, out, width, height, nullptr);
    timer.stop();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}

// ---------------------------------------------------------------------------
// Auto-exposure metering with the reference's launchers
// (src/Cuda/JuicerCudaAutoExposure.cu:667 juicer_cuda_auto_exposure_meter_to_device,
// :864 juicer_cuda_auto_exposure_build_center_weight_tables), driven as
// src/Cuda/JuicerCudaExecutor.cpp:1018-1070 meter_camera_exposure does: the film raw
// and reconstruction payloads of the recipe, the preview descriptor of the record,
// weight tables for centre-weighted metering. `src` is the device address of the
// source image's bounds origin. Writes the float scale to *scale_out. Synchronous.
// Returns 0, or the launcher's non-zero code (+100), or a cudaError_t (+1000).
// ---------------------------------------------------------------------------
#include "Cuda/JuicerCudaResources.h"

extern "C" int ref_auto_exposure(const FjPreparedHostData* h, const float* const* lut, const FjAutoExposure* m,
                                 const float* src, long src_row_bytes, int comps, float* scale_out) {
    Arena a;
    unsigned* d_flags = nullptr;
    if (cudaMalloc(&d_flags, sizeof(unsigned)) != cudaSuccess) return 1002;
    a.ptrs.push_back(d_flags);
    JuicerCuda::PipelineRunParams p;
    if (!pack(*h, lut, a, p, d_flags)) return 1;
    JuicerCuda::AutoExposurePreviewDescriptor d{};
    d.sourceX1 = m->source_bounds.x1;
    d.sourceY1 = m->source_bounds.y1;
    d.sourceX2 = m->source_bounds.x2;
    d.sourceY2 = m->source_bounds.y2;
    d.meterX1 = m->meter_bounds.x1;
    d.meterY1 = m->meter_bounds.y1;
    d.meterX2 = m->meter_bounds.x2;
    d.meterY2 = m->meter_bounds.y2;
    d.previewWidth = m->preview_width;
    d.previewHeight = m->preview_height;
    d.method = static_cast<Spektrafilm::AutoExposureMethod>(m->method);
    d.hash = m->hash;
    JuicerCuda::AutoExposureSourceFormat fmt{};
    fmt.componentCount = comps;
    fmt.filmRaw = p.filmRaw;
    fmt.reconstruction = p.filmExpose.reconstruction;
    const int gx = (d.previewWidth + 15) / 16, gy = (d.previewHeight + 15) / 16;
    const int blocks = gx > 0 && gy > 0 ? gx * gy : 1;
    JuicerCudaAutoExposureScratch scratch{};
    void* mem[6] = {};
    const size_t sizes[6] = {sizeof(JuicerCudaAutoExposurePartial) * (size_t)blocks,
                             sizeof(JuicerCudaAutoExposurePartial) * (size_t)blocks, sizeof(unsigned),
                             sizeof(unsigned) * 2048, sizeof(float) * (size_t)(d.previewWidth > 0 ? d.previewWidth : 1),
                             sizeof(float) * (size_t)(d.previewHeight > 0 ? d.previewHeight : 1)};
    for (int i = 0; i < 6; ++i) {
        if (cudaMalloc(&mem[i], sizes[i]) != cudaSuccess) return 1002;
        a.ptrs.push_back(mem[i]);
    }
    scratch.partialsA = static_cast<JuicerCudaAutoExposurePartial*>(mem[0]);
    scratch.partialsB = static_cast<JuicerCudaAutoExposurePartial*>(mem[1]);
    scratch.partialCapacity = blocks;
    scratch.maxYBits = static_cast<unsigned*>(mem[2]);
    scratch.histogram = static_cast<unsigned*>(mem[3]);
    scratch.weightsX = static_cast<float*>(mem[4]);
    scratch.weightsY = static_cast<float*>(mem[5]);
    float* d_scale = nullptr;
    if (cudaMalloc(&d_scale, sizeof(float)) != cudaSuccess) return 1002;
    a.ptrs.push_back(d_scale);
    JuicerCudaAutoExposureDeviceState state{};
    state.exposureScale = d_scale;
    const char* why = nullptr;
    if (m->method == FJ_METER_CENTER_WEIGHTED && d.previewWidth > 0 && d.previewHeight > 0) {
        const int rc = juicer_cuda_auto_exposure_build_center_weight_tables(d.previewWidth, d.previewHeight,
                                                                            scratch.weightsX, scratch.weightsY,
                                                                            nullptr, &why);
        if (rc != 0) return 100 + rc;
    }
    const int rc = juicer_cuda_auto_exposure_meter_to_device(src, (size_t)src_row_bytes, d, fmt, scratch, state,
                                                             nullptr, &why);
    if (rc != 0) return 100 + rc;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(scale_out, d_scale, sizeof(float), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : 1000 + (int)e;
}

// ---------------------------------------------------------------------------
// Enlarger diffusion stages with the reference's launchers
// (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2924 print-linear exposure, :2943 print
// development from the diffused planes). stage 0: density planes in0..2 (C, M, Y) ->
// linear planes out0..2 (C-, M-, Y-forming), dust may be NULL; stage 1: linear planes
// in0..2 -> print density out0..2. Device pointers, width-stride planes. Synchronous.
// ---------------------------------------------------------------------------
extern "C" cudaError_t juicer_cuda_print_focused_enlarger_linear_exposure(
    const JuicerCuda::PrintPipelineRunParams*, const float*, const float*, const float*,
    JuicerCuda::EnlargerPrintLinearExposurePlanes, const float*, void*);
extern "C" cudaError_t juicer_cuda_print_focused_develop_from_enlarger_linear(
    const JuicerCuda::PrintPipelineRunParams*, JuicerCuda::EnlargerPrintLinearExposurePlanes, float*, float*, float*,
    void*);

extern "C" int ref_enlarger(const FjPreparedHostData* h, const float* const* lut, int stage, float* in0, float* in1,
                            float* in2, const float* dust, int width, int height, float* out0, float* out1,
                            float* out2) {
    Arena a;
    unsigned* d_flags = nullptr;
    if (cudaMalloc(&d_flags, sizeof(unsigned)) != cudaSuccess) return 2;
    cudaMemset(d_flags, 0, sizeof(unsigned));
    a.ptrs.push_back(d_flags);
    JuicerCuda::PipelineRunParams p;
    if (!pack(*h, lut, a, p, d_flags)) return 1;
    JuicerCuda::PrintPipelineRunParams q{};
    q.src = in0;
    q.srcRowBytes = (size_t)width * sizeof(float);
    q.dst = out0;
    q.dstRowBytes = (size_t)width * sizeof(float);
    q.width = width;
    q.height = height;
    q.nComponents = 3;
    q.filmExpose = p.filmExpose;
    q.filmDevelop = p.filmDevelop;
    q.printExpose = p.printExpose;
    q.printDevelop = p.printDevelop;
    q.scanStage = p.scanStage;
    q.filmRaw = p.filmRaw;
    JuicerCuda::EnlargerPrintLinearExposurePlanes planes{};
    planes.rowStrideFloats = (size_t)width;
    cudaError_t e;
    if (stage == 0) {
        planes.redSensitiveCForming = out0;
        planes.greenSensitiveMForming = out1;
        planes.blueSensitiveYForming = out2;
        e = juicer_cuda_print_focused_enlarger_linear_exposure(&q, in0, in1, in2, planes, dust, nullptr);
    } else {
        planes.redSensitiveCForming = in0;
        planes.greenSensitiveMForming = in1;
        planes.blueSensitiveYForming = in2;
        e = juicer_cuda_print_focused_develop_from_enlarger_linear(&q, planes, out0, out1, out2, nullptr);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return (int)e;
}
