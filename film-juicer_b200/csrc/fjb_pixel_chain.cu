// fjb_pixel_chain.cu -- the fused per-pixel film-process kernel (a1..a13).
//
// One persistent launch walks the frame with a grid-stride loop (grid sized to the
// SM count times the variant's resident CTAs per SM). Each CTA stages the recipe's density curves into shared memory once;
// the print spectral coefficients are kernel parameters (constant bank); the TC LUT,
// scanner nodes and gamut boundary are 16-byte-vector reads through L1/L2.
//
// Variants (template flags) cover the reference's fused kernels
// (src/Cuda/Scan/JuicerCudaScanPipeline.cu:1700-1868 pipeline_direct/carrier_kernel,
// :1891 focused_capture_film_density_kernel, :1944 scan_linear_density_rgb_kernel,
// :1362 develop_print_density_kernel):
//   Input  = source RGB(A) | carrier planes (B, G, R linear exposure) | density planes
//   Output = encoded RGB(A) | capture density planes (C, M, Y) | linear output-RGB
//            planes (for the scanner post effects, then encode_planes_kernel)
#include <cuda_runtime.h>

#include "fjb_internal.h"
#include "fjb_pixel_math.cuh"
#include "fjb_launches.h"

namespace fjb {

enum InputKind : int { kInSource = 0, kInCarrier = 1, kInDensity = 2, kInPrintRaw = 3 };
enum OutputKind : int {
    kOutEncoded = 0,
    kOutDensity = 1,
    kOutDirSource = 2,
    kOutLinearRgb = 3,
    kOutPrintRaw = 4,
    kOutEnlargerLinear = 5,  // print-linear exposure planes before the enlarger diffusion
    kOutEnlargerDevelop = 6, // print density from the diffused print-linear exposure
};

// Spatial-DIR source (src/Cuda/Film/JuicerCudaFilmPipeline.cu:124-214): raw log
// exposure, pre-DIR layer densities and the donor corrections they release.
__device__ __forceinline__ void dir_source(const PixelParams& p, const float* __restrict__ blob, const float e[3],
                                           long long idx) {
    float logE[3], layer[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        logE[c] = log_exposure(e[c]);
        const float s = clamp_infinite_log(blob, p.film_curve[c], logE[c]);
        layer[c] = curve_sample(blob, p.film_curve[c], s, p.gamma_bgr[c]);
    }
    float corr[3];
    const unsigned fail = dir_donor_corrections(p, layer, corr);
    flag_dir_failure(p, fail);
    p.dir_src_y[idx] = corr[0];
    p.dir_src_m[idx] = corr[1];
    p.dir_src_c[idx] = corr[2];
    p.dir_src_log_b[idx] = logE[0];
    p.dir_src_log_g[idx] = logE[1];
    p.dir_src_log_r[idx] = logE[2];
}

template <int In, int Out, bool Print, bool SpatialDir>
__global__ void __launch_bounds__(kPixelThreads) pixel_chain_kernel(const __grid_constant__ PixelParams p) {
    extern __shared__ float4 smem4[];
    float* blob = reinterpret_cast<float*>(smem4);
    {
        const float4* g = reinterpret_cast<const float4*>(p.curve_blob);
        const int n4 = p.curve_blob_floats >> 2;
        for (int i = threadIdx.x; i < n4; i += blockDim.x) smem4[i] = __ldg(g + i);
    }
    __syncthreads();

    const long long total = (long long)p.width * (long long)p.height;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
        const int y = (int)(idx / p.width);
        const int x = (int)(idx - (long long)y * p.width);
        const float* srcPix = nullptr;
        if (p.src) {
            srcPix = reinterpret_cast<const float*>(p.src + (long long)y * p.src_row_bytes) + (long long)x * p.components;
        }

        if constexpr (Out == kOutDirSource) {
            float e[3];
            if constexpr (In == kInCarrier) {
                const long long ci = (long long)y * p.carrier_stride + x;
                e[0] = p.carrier_b[ci];
                e[1] = p.carrier_g[ci];
                e[2] = p.carrier_r[ci];
                for (int c = 0; c < 3; ++c) e[c] = fmaxf(0.0f, e[c] * p.route_correction_scale);
            } else {
                const float in[3] = {srcPix[0], srcPix[1], srcPix[2]};
                camera_linear_exposure(p, in, true, e);
            }
            dir_source(p, blob, e, idx);
            continue;
        }

        float d[3];
        if constexpr (In == kInDensity) {
            d[0] = p.scan_density_c[idx];
            d[1] = p.scan_density_m[idx];
            d[2] = p.scan_density_y[idx];
        } else if constexpr (In == kInPrintRaw) {
            // print development from the spectral integral of the tensor-core form
            float raw[3] = {p.print_raw_c[idx], p.print_raw_m[idx], p.print_raw_y[idx]};
            print_finish(p, blob, raw, d, p.film_dust ? p.film_dust[idx] : 1.0f);
        } else if constexpr (SpatialDir) {
            float logRaw[3];
            if (p.dir_log_raw_b) {
                logRaw[0] = __ldg(p.dir_log_raw_b + idx);
                logRaw[1] = __ldg(p.dir_log_raw_g + idx);
                logRaw[2] = __ldg(p.dir_log_raw_r + idx);
            } else {
                float e[3];
                if constexpr (In == kInCarrier) {
                    const long long ci = (long long)y * p.carrier_stride + x;
                    e[0] = p.carrier_b[ci];
                    e[1] = p.carrier_g[ci];
                    e[2] = p.carrier_r[ci];
                    for (int c = 0; c < 3; ++c) e[c] = fmaxf(0.0f, e[c] * p.route_correction_scale);
                } else {
                    const float in[3] = {srcPix[0], srcPix[1], srcPix[2]};
                    camera_linear_exposure(p, in, true, e);
                }
                for (int c = 0; c < 3; ++c) logRaw[c] = log_exposure(e[c]);
            }
            float corr[3] = {p.dir_filtered_y[idx], p.dir_filtered_m[idx], p.dir_filtered_c[idx]};
            develop_capture_spatial(p, blob, logRaw, corr, d);
        } else {
            float e[3];
            if constexpr (In == kInCarrier) {
                const long long ci = (long long)y * p.carrier_stride + x;
                e[0] = p.carrier_b[ci];
                e[1] = p.carrier_g[ci];
                e[2] = p.carrier_r[ci];
                for (int c = 0; c < 3; ++c) e[c] = fmaxf(0.0f, e[c] * p.route_correction_scale);
            } else {
                const float in[3] = {srcPix[0], srcPix[1], srcPix[2]};
                camera_linear_exposure(p, in, true, e);
            }
            develop_capture(p, blob, e, d);
        }

        if constexpr (Out == kOutDensity) {
            p.density_c[idx] = d[0];
            p.density_m[idx] = d[1];
            p.density_y[idx] = d[2];
            continue;
        }

        if constexpr (Out == kOutEnlargerLinear) {
            // src/Cuda/Scan/JuicerCudaScanPipeline.cu:1392-1447 with print_inner_raw_device and
            // print_linear_for_diffusion_device (src/Cuda/JuicerCudaDeviceHelpers.cuh:966-1010)
            float raw[3];
            print_spectral(p.spectral, d, raw);
            float lin[3];
            enlarger_linear(p, raw, p.film_dust ? p.film_dust[idx] : 1.0f, lin);
            p.lin_r[idx] = lin[0];
            p.lin_g[idx] = lin[1];
            p.lin_b[idx] = lin[2];
            continue;
        }
        if constexpr (Out == kOutEnlargerDevelop) {
            // :1449-1488 with print_log_encode_diffused_device (:1025) and the print curves
            for (int c = 0; c < 3; ++c) d[c] = curve_sample(blob, p.print_curve[c], log10f(fmaxf(d[c], 0.0f) + 1e-10f), 1.0f);
            p.density_c[idx] = d[0];
            p.density_m[idx] = d[1];
            p.density_y[idx] = d[2];
            continue;
        }
        if constexpr (Out == kOutPrintRaw) {
            float raw[3];
            print_spectral(p.spectral, d, raw);
            p.lin_r[idx] = raw[0];
            p.lin_g[idx] = raw[1];
            p.lin_b[idx] = raw[2];
            continue;
        }
        if constexpr (Print) {
            print_develop(p, blob, d, p.film_dust ? p.film_dust[idx] : 1.0f);
        }
        // the direct route scans the film itself: its dust darkens the scanned XYZ
        const float* dust = !Print && In != kInPrintRaw && p.film_dust ? p.film_dust + idx : nullptr;

        double rgb[3];
        if constexpr (Out == kOutLinearRgb) {
            // src/Cuda/Scan/JuicerCudaScanPipeline.cu:1944-2037 scan_linear_density_rgb_kernel
            const float glare = p.scan_glare ? p.scan_glare[idx] : -1.0f;
            if (!scan_to_linear(p, d, rgb, glare, dust)) {
                flag_scan_failure(p);
                rgb[0] = rgb[1] = rgb[2] = 0.0;
            }
            p.lin_r[idx] = (float)rgb[0];
            p.lin_g[idx] = (float)rgb[1];
            p.lin_b[idx] = (float)rgb[2];
            continue;
        }
        float* dstPix = reinterpret_cast<float*>(p.dst + (long long)y * p.dst_row_bytes) + (long long)x * p.components;
        if (!scan_to_linear(p, d, rgb, -1.0f, dust)) {
            flag_scan_failure(p);
            dstPix[0] = 0.0f;
            dstPix[1] = 0.0f;
            dstPix[2] = 0.0f;
            if (p.components == 4) dstPix[3] = srcPix ? srcPix[3] : 1.0f;
            continue;
        }
        encode_output(p, rgb);
        dstPix[0] = (float)rgb[0];
        dstPix[1] = (float)rgb[1];
        dstPix[2] = (float)rgb[2];
        if (p.components == 4) dstPix[3] = srcPix ? srcPix[3] : 1.0f;
    }
}

// Mitchell (B = C = 1/3) sample of a plane at (x, y), clamped to the edge, summed in
// FP64 (src/Cuda/Scan/JuicerCudaScanPipeline.cu:1514-1556).
__device__ float plane_mitchell(const float* __restrict__ plane, int width, int height, float x, float y) {
    x = fminf(fmaxf(x, 0.0f), (float)(width - 1));
    y = fminf(fmaxf(y, 0.0f), (float)(height - 1));
    const int ix = (int)floorf(x), iy = (int)floorf(y);
    const float tx = x - (float)ix, ty = y - (float)iy;
    const float wx[4] = {mitchell(tx + 1.0f), mitchell(tx), mitchell(tx - 1.0f), mitchell(tx - 2.0f)};
    const float wy[4] = {mitchell(ty + 1.0f), mitchell(ty), mitchell(ty - 1.0f), mitchell(ty - 2.0f)};
    double acc = 0.0;
    for (int j = 0; j < 4; ++j) {
        const int sy = min(max(iy + j - 1, 0), height - 1);
        const double wyj = wy[j];
        const float* row = plane + (size_t)sy * width;
        for (int i = 0; i < 4; ++i) {
            const int sx = min(max(ix + i - 1, 0), width - 1);
            acc += wyj * wx[i] * (double)__ldg(row + sx);
        }
    }
    return (float)acc;
}

// Bilinear sample of the gate mask, clamped (src/Cuda/Scan/JuicerCudaScanPipeline.cu:1331-1360).
__device__ float gate_sample(const float* __restrict__ mask, int width, int height, float x, float y) {
    const float fx = fminf(fmaxf(x, 0.0f), (float)(width - 1));
    const float fy = fminf(fmaxf(y, 0.0f), (float)(height - 1));
    const int x0 = (int)floorf(fx), y0 = (int)floorf(fy);
    const int x1 = x0 + 1 < width ? x0 + 1 : x0;
    const int y1 = y0 + 1 < height ? y0 + 1 : y0;
    const float tx = fx - (float)x0, ty = fy - (float)y0;
    const float m00 = __ldg(mask + y0 * width + x0), m10 = __ldg(mask + y0 * width + x1);
    const float m01 = __ldg(mask + y1 * width + x0), m11 = __ldg(mask + y1 * width + x1);
    const float m0 = m00 + (m10 - m00) * tx;
    const float m1 = m01 + (m11 - m01) * tx;
    return m0 + (m1 - m0) * ty;
}

// Encoding of linear output-RGB planes (src/Cuda/Scan/JuicerCudaScanPipeline.cu:2096-2182
// focused_scan_output_encode_kernel): with gate weave the planes are resampled along the
// frame's shift and rotation about its centre; the gate mask multiplies the result.
__global__ void __launch_bounds__(kPixelThreads) encode_planes_kernel(const __grid_constant__ PixelParams p) {
    const long long total = (long long)p.width * (long long)p.height;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
        const int y = (int)(idx / p.width);
        const int x = (int)(idx - (long long)y * p.width);
        double rgb[3];
        if (p.weave_active) {
            const float cx = 0.5f * (float)(p.width - 1), cy = 0.5f * (float)(p.height - 1);
            const float ox = (float)x - cx, oy = (float)y - cy;
            const float sx = p.weave_cos * ox - p.weave_sin * oy + cx + p.weave_dx;
            const float sy = p.weave_sin * ox + p.weave_cos * oy + cy + p.weave_dy;
            rgb[0] = plane_mitchell(p.lin_r, p.width, p.height, sx, sy);
            rgb[1] = plane_mitchell(p.lin_g, p.width, p.height, sx, sy);
            rgb[2] = plane_mitchell(p.lin_b, p.width, p.height, sx, sy);
        } else {
            rgb[0] = (double)p.lin_r[idx];
            rgb[1] = (double)p.lin_g[idx];
            rgb[2] = (double)p.lin_b[idx];
        }
        if (p.gate_mask && p.gate_w > 0 && p.gate_h > 0) {
            const double t = (double)gate_sample(p.gate_mask, p.gate_w, p.gate_h, (float)(p.roi_x + x) * 0.5f - 0.25f,
                                                 (float)(p.roi_y + y) * 0.5f - 0.25f);
            rgb[0] *= t;
            rgb[1] *= t;
            rgb[2] *= t;
        }
        encode_output(p, rgb);
        float* dstPix = reinterpret_cast<float*>(p.dst + (long long)y * p.dst_row_bytes) + (long long)x * p.components;
        dstPix[0] = (float)rgb[0];
        dstPix[1] = (float)rgb[1];
        dstPix[2] = (float)rgb[2];
        if (p.components == 4) {
            const float* srcPix =
                reinterpret_cast<const float*>(p.src + (long long)y * p.src_row_bytes) + (long long)x * p.components;
            dstPix[3] = srcPix[3];
        }
    }
}


// Camera linear exposure (no route correction) into planar B, G, R carrier planes.
__global__ void __launch_bounds__(kPixelThreads) camera_exposure_kernel(const __grid_constant__ PixelParams p,
                                                                        float* b, float* g, float* r,
                                                                        long long stride) {
    const long long total = (long long)p.width * (long long)p.height;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += step) {
        const int y = (int)(idx / p.width);
        const int x = (int)(idx - (long long)y * p.width);
        const float* s = reinterpret_cast<const float*>(p.src + (long long)y * p.src_row_bytes) + (long long)x * p.components;
        const float in[3] = {s[0], s[1], s[2]};
        float e[3];
        camera_linear_exposure(p, in, false, e);
        const long long o = (long long)y * stride + x;
        b[o] = e[0];
        g[o] = e[1];
        r[o] = e[2];
    }
}

// Grid of a grid-stride pixel kernel: every CTA the device holds at once (the kernel's
// own occupancy at kPixelThreads threads and `smem` bytes of shared memory, so kernels
// with few registers fill the SMs), or one CTA per 256 pixels when that is fewer.
static int persistent_grid(long long total, const void* kernel, size_t smem) {
    int device = 0;
    cudaGetDevice(&device);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (sms <= 0) sms = 148;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPixelThreads, smem) != cudaSuccess ||
        per_sm <= 0) {
        cudaGetLastError(); // the query's own failure is not the launch's
        per_sm = kPixelBlocksPerSm;
    }
    const long long blocksNeeded = (total + kPixelThreads - 1) / kPixelThreads;
    const long long cap = (long long)sms * per_sm;
    return (int)(blocksNeeded < cap ? blocksNeeded : cap);
}

template <int In, int Out, bool Print, bool SpatialDir>
static cudaError_t launch_variant(const PixelParams& p, long long total, size_t smem, cudaStream_t stream) {
    auto* k = pixel_chain_kernel<In, Out, Print, SpatialDir>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int grid = persistent_grid(total, reinterpret_cast<const void*>(k), smem);
    fjb::count_launch();
    k<<<grid, kPixelThreads, smem, stream>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_camera_exposure(const PixelParams& p, float* b, float* g, float* r, long long stride,
                                   cudaStream_t stream) {
    const long long total = (long long)p.width * (long long)p.height;
    if (total <= 0) return cudaSuccess;
    fjb::count_launch();
    camera_exposure_kernel<<<persistent_grid(total, reinterpret_cast<const void*>(camera_exposure_kernel), 0),
                             kPixelThreads, 0, stream>>>(p, b, g, r, stride);
    return cudaGetLastError();
}

cudaError_t launch_pixel_chain(const PixelParams& p, PixelStage stage, cudaStream_t stream) {
    const long long total = (long long)p.width * (long long)p.height;
    if (total <= 0) return cudaSuccess;
    if (p.route == kRoutePrint && p.print_form != kPrintFp32 && !p.print_done &&
        (stage == PixelStage::DensityToOutput || stage == PixelStage::DensityToLinearRgb ||
         stage == PixelStage::DensityToPrintRaw))
        return launch_print_tensor(p, stage, stream);
    if ((p.curve_blob_floats & 3) != 0) return cudaErrorInvalidValue;
    const size_t smem = (size_t)p.curve_blob_floats * sizeof(float);
    const bool print = p.route == kRoutePrint && !p.print_done; // enlarger diffusion: scan the print density
    const bool sdir = p.dir_spatial != 0;
    switch (stage) {
        case PixelStage::SourceToOutput:
            if (sdir) return print ? launch_variant<kInSource, kOutEncoded, true, true>(p, total, smem, stream)
                                   : launch_variant<kInSource, kOutEncoded, false, true>(p, total, smem, stream);
            return print ? launch_variant<kInSource, kOutEncoded, true, false>(p, total, smem, stream)
                         : launch_variant<kInSource, kOutEncoded, false, false>(p, total, smem, stream);
        case PixelStage::CarrierToOutput:
            if (sdir) return print ? launch_variant<kInCarrier, kOutEncoded, true, true>(p, total, smem, stream)
                                   : launch_variant<kInCarrier, kOutEncoded, false, true>(p, total, smem, stream);
            return print ? launch_variant<kInCarrier, kOutEncoded, true, false>(p, total, smem, stream)
                         : launch_variant<kInCarrier, kOutEncoded, false, false>(p, total, smem, stream);
        case PixelStage::SourceToDensity:
            return sdir ? launch_variant<kInSource, kOutDensity, false, true>(p, total, smem, stream)
                        : launch_variant<kInSource, kOutDensity, false, false>(p, total, smem, stream);
        case PixelStage::CarrierToDensity:
            return sdir ? launch_variant<kInCarrier, kOutDensity, false, true>(p, total, smem, stream)
                        : launch_variant<kInCarrier, kOutDensity, false, false>(p, total, smem, stream);
        case PixelStage::SourceToDirSource:
            return launch_variant<kInSource, kOutDirSource, false, false>(p, total, smem, stream);
        case PixelStage::CarrierToDirSource:
            return launch_variant<kInCarrier, kOutDirSource, false, false>(p, total, smem, stream);
        case PixelStage::DensityToLinearRgb:
            return print ? launch_variant<kInDensity, kOutLinearRgb, true, false>(p, total, smem, stream)
                         : launch_variant<kInDensity, kOutLinearRgb, false, false>(p, total, smem, stream);
        case PixelStage::LinearRgbToOutput:
            fjb::count_launch();
            encode_planes_kernel<<<persistent_grid(total, reinterpret_cast<const void*>(encode_planes_kernel), 0),
                                   kPixelThreads, 0, stream>>>(p);
            return cudaGetLastError();
        case PixelStage::DensityToOutput:
            return print ? launch_variant<kInDensity, kOutEncoded, true, false>(p, total, smem, stream)
                         : launch_variant<kInDensity, kOutEncoded, false, false>(p, total, smem, stream);
        case PixelStage::DensityToPrintRaw:
            return launch_variant<kInDensity, kOutPrintRaw, true, false>(p, total, smem, stream);
        case PixelStage::DensityToEnlargerLinear:
            return launch_variant<kInDensity, kOutEnlargerLinear, true, false>(p, total, smem, stream);
        case PixelStage::EnlargerLinearToPrintDensity:
            return launch_variant<kInDensity, kOutEnlargerDevelop, false, false>(p, total, smem, stream);
        case PixelStage::RawToOutput:
            return launch_variant<kInPrintRaw, kOutEncoded, false, false>(p, total, smem, stream);
        case PixelStage::RawToLinearRgb:
            return launch_variant<kInPrintRaw, kOutLinearRgb, false, false>(p, total, smem, stream);
    }
    return cudaErrorInvalidValue;
}

} // namespace fjb
