// fjb_print_tc.cu -- the print stage with its 81-wavelength contraction on the
// fifth-generation tensor cores (tcgen05, sm_100a only).
//
// Reference: print_spectral_integrate_device (src/Cuda/JuicerCudaDeviceHelpers.cuh:866-935)
//   D(l) = sum_c d_c eps_c(l) + base(l),  T(l) = 10^-D(l) I_filt(l),  raw_c = sum_l T(l) S_c(l).
// The recipe folds it into nd(l) = -(eps_c, eps_m, eps_y, base)(l) log2(10) and
// sens(l) = S(l) I_filt(l) (fjb_params.h), so T(l) = 2^(d . nd(l) + nd3(l)) and
// raw_c = sum_l T(l) sens_c(l).
//
// One CTA of 128 threads takes tiles of 128 consecutive pixels (one per thread, one
// TMEM lane per pixel):
//   GEMM1  D1[128 x 96] = A1[128 x 16] B1[96 x 16]^T  (M = pixels, N = wavelengths
//          padded 81 -> 96, K = 16). A1 row = (d_hi[3], d_lo[3], d_hi[3], 1, 1, 0...),
//          B1 row = (nd_hi[3], nd_hi[3], nd_lo[3], nd3_hi, nd3_lo, 0...): BF16 hi + lo
//          pairs of both sides, so d . nd + nd3 is carried to about 2^-17 relative
//          (only d_lo nd_lo is dropped), accumulated in FP32 in TMEM.
//   exp2   per pixel and wavelength in FP32 on the MUFU, read from TMEM with
//          tcgen05.ld; T rounded to BF16 (kPrintTensor) or to a BF16 pair hi + lo
//          (kPrintTensorSplit) into shared memory.
//   GEMM2  D2[128 x 16] = T[128 x 96] [sens_hi; sens_lo][16 x 96]^T (+ T_lo sens_hi),
//          six K-steps of 16 per product, FP32 accumulate; columns 0..2 are raw C, M, Y.
//   then   the print development, scan and output encoding of each pixel in FP32,
//          the same device functions as the FP32 kernel (fjb_pixel_math.cuh).
// Pixels with a non-finite density (failed DIR) take the FP32 cold path for raw.
//
// Operand tiles in shared memory are K-major without swizzle: 8-row x 16-byte core
// matrices, the two 8-element K chunks of a K-step 128 B apart (leading byte offset),
// 8-row groups K/8 x 128 B apart (stride byte offset). One thread issues the MMAs;
// completion is signalled by tcgen05.commit to an mbarrier that every thread waits
// on with an iteration limit (on expiry the kernel sets kErrTensorWait, frees its
// TMEM and returns).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fjb_internal.h"
#include "fjb_launches.h"
#include "fjb_pixel_math.cuh"

namespace fjb {

namespace {

constexpr int kTcThreads = 128;     // pixels per tile = MMA M = TMEM lanes
constexpr int kTcLambda = 96;       // 81 wavelengths padded to six K-steps of 16
constexpr int kTcK1 = 16;           // GEMM1 K
constexpr uint32_t kTmemCols = 128; // D1 in columns 0..95, D2 in 96..111
constexpr uint32_t kD2Col = 96;

// shared-memory map, bytes from the (128-aligned) dynamic base
constexpr uint32_t kOffA1 = 0;       // 128 x 16 BF16
constexpr uint32_t kOffB1 = 4096;    // 96 x 16 BF16 (3072 B)
constexpr uint32_t kOffB2 = 7168;    // 16 x 96 BF16 sens hi (3072 B), then sens lo
constexpr uint32_t kOffA2 = 13312;   // 128 x 96 BF16 T hi (24576 B)
constexpr uint32_t kOffA2lo = 37888; // 128 x 96 BF16 T lo (split form only)
__host__ __device__ constexpr uint32_t off_bar(bool split) { return split ? 62464u : 37888u; }
__host__ __device__ constexpr uint32_t off_blob(bool split) { return off_bar(split) + 64u; }

// Byte offset of element (row, k) in a K-major, no-swizzle operand with `kdim` columns.
__host__ __device__ constexpr uint32_t kmajor(int row, int k, int kdim) {
    return (uint32_t)((row >> 3) * (kdim / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (tcgen05): start >> 4 in bits 0..13, leading byte
// offset >> 4 in 16..29, stride byte offset >> 4 in 32..45, descriptor version 1 in
// 46..47, no swizzle (bits 61..63 = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4..5 = 1), BF16 A and B
// (bits 7..9 and 10..12 = 1), both K-major, N >> 3 in bits 17..22, M >> 4 in 24..28.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Bounded wait for the mbarrier phase `parity`; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < (1 << 20); ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane (load and wait in one block).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo_k, float hi_k) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo_k, hi_k); // .x (even k) in the low half
    return *reinterpret_cast<const uint32_t*>(&v);
}

// hi = BF16(v), lo = BF16(v - hi); a non-finite v keeps its value in hi and 0 in lo.
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(isfinite(v) ? v - __bfloat162float(hi) : 0.0f);
}

template <int Out, bool Split>
__global__ void __launch_bounds__(kTcThreads) print_tc_kernel(const __grid_constant__ PixelParams p) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const uint32_t sbase = smem_addr(tc_smem);
    float* blob = reinterpret_cast<float*>(tc_smem + off_blob(Split));
    uint64_t* bars = reinterpret_cast<uint64_t*>(tc_smem + off_bar(Split));
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + off_bar(Split) + 16);
    const uint32_t bar1 = smem_addr(bars), bar2 = smem_addr(bars + 1);

    // curves into shared memory
    {
        const float4* g = reinterpret_cast<const float4*>(p.curve_blob);
        float4* s4 = reinterpret_cast<float4*>(blob);
        const int n4 = p.curve_blob_floats >> 2;
        for (int i = tid; i < n4; i += kTcThreads) s4[i] = __ldg(g + i);
    }
    // B1: per wavelength (nd_hi[3], nd_hi[3], nd_lo[3], nd3_hi, nd3_lo, 0 x 5)
    const int count = p.spectral.count;
    for (int l = tid; l < kTcLambda; l += kTcThreads) {
        __nv_bfloat16 row[kTcK1];
        for (int k = 0; k < kTcK1; ++k) row[k] = __float2bfloat16_rn(0.0f);
        if (l < count) {
            for (int c = 0; c < 3; ++c) {
                __nv_bfloat16 hi, lo;
                split_bf16(p.spectral.nd[l][c], hi, lo);
                row[c] = hi;
                row[3 + c] = hi;
                row[6 + c] = lo;
            }
            split_bf16(p.spectral.nd[l][3], row[9], row[10]);
        }
        for (int k = 0; k < kTcK1; ++k)
            *reinterpret_cast<__nv_bfloat16*>(tc_smem + kOffB1 + kmajor(l, k, kTcK1)) = row[k];
    }
    // B2: sens hi and lo, rows C, M, Y then zeros, K = wavelength
    for (int e = tid; e < 16 * kTcLambda; e += kTcThreads) {
        const int n = e / kTcLambda, l = e - n * kTcLambda;
        __nv_bfloat16 hi = __float2bfloat16_rn(0.0f), lo = hi;
        if (n < 3 && l < count) split_bf16(p.spectral.sens[l][n], hi, lo);
        *reinterpret_cast<__nv_bfloat16*>(tc_smem + kOffB2 + kmajor(n, l, kTcLambda)) = hi;
        *reinterpret_cast<__nv_bfloat16*>(tc_smem + kOffB2 + 3072 + kmajor(n, l, kTcLambda)) = lo;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar2) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);

    const uint64_t dA1 = smem_desc(sbase + kOffA1, 128, 256);
    const uint64_t dB1 = smem_desc(sbase + kOffB1, 128, 256);
    const uint32_t i1 = idesc_bf16(128, kTcLambda);
    const uint32_t i2 = idesc_bf16(128, 16);

    const long long total = (long long)p.width * (long long)p.height;
    const long long tiles = (total + kTcThreads - 1) / kTcThreads;
    uint32_t phase = 0;
    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long idx = tile * kTcThreads + tid;
        const bool live = idx < total;
        float d[3] = {0.0f, 0.0f, 0.0f};
        if (live) {
            d[0] = p.scan_density_c[idx];
            d[1] = p.scan_density_m[idx];
            d[2] = p.scan_density_y[idx];
        }
        const bool finite = live && isfinite(d[0]) && isfinite(d[1]) && isfinite(d[2]);
        {
            __nv_bfloat16 a[kTcK1];
            for (int k = 0; k < kTcK1; ++k) a[k] = __float2bfloat16_rn(0.0f);
            if (finite) {
                for (int c = 0; c < 3; ++c) {
                    __nv_bfloat16 hi, lo;
                    split_bf16(d[c], hi, lo);
                    a[c] = hi;
                    a[3 + c] = lo;
                    a[6 + c] = hi;
                }
                a[9] = a[10] = __float2bfloat16_rn(1.0f);
            }
            *reinterpret_cast<uint4*>(tc_smem + kOffA1 + kmajor(tid, 0, kTcK1)) = *reinterpret_cast<const uint4*>(a);
            *reinterpret_cast<uint4*>(tc_smem + kOffA1 + kmajor(tid, 8, kTcK1)) =
                *reinterpret_cast<const uint4*>(a + 8);
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        if (tid == 0) {
            fence_after();
            mma_bf16(tmem, dA1, dB1, i1, 0u);
            mma_commit(bar1);
        }
        // every thread waits; the CTA goes on only if all saw the MMA complete
        bool ok = __syncthreads_and(mbar_wait(bar1, phase)) != 0;
        fence_after();
        if (ok) {
            // T = 2^D for the 96 columns of this pixel, as BF16 (and BF16 remainders)
#pragma unroll
            for (int chunk = 0; chunk < 3; ++chunk) {
                uint32_t r[32];
                tmem_ld32(lane_base + (uint32_t)(chunk * 32), r);
                uint32_t hi[16], lo[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const float t0 = mufu_exp2(__uint_as_float(r[2 * j]));
                    const float t1 = mufu_exp2(__uint_as_float(r[2 * j + 1]));
                    hi[j] = pack_bf16(t0, t1);
                    if constexpr (Split) {
                        const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&hi[j]);
                        lo[j] = pack_bf16(t0 - __low2float(h), t1 - __high2float(h));
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t off = kmajor(tid, chunk * 32 + q * 8, kTcLambda);
                    *reinterpret_cast<uint4*>(tc_smem + kOffA2 + off) =
                        make_uint4(hi[4 * q], hi[4 * q + 1], hi[4 * q + 2], hi[4 * q + 3]);
                    if constexpr (Split)
                        *reinterpret_cast<uint4*>(tc_smem + kOffA2lo + off) =
                            make_uint4(lo[4 * q], lo[4 * q + 1], lo[4 * q + 2], lo[4 * q + 3]);
                }
            }
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        if (!ok) {
            if (tid == 0 && p.error_flags) atomicOr(p.error_flags, kErrTensorWait);
            break;
        }
        if (tid == 0) {
            fence_after();
#pragma unroll
            for (int j = 0; j < 6; ++j)
                mma_bf16(tmem + kD2Col, smem_desc(sbase + kOffA2 + 256u * j, 128, 1536),
                         smem_desc(sbase + kOffB2 + 256u * j, 128, 1536), i2, j > 0 ? 1u : 0u);
#pragma unroll
            for (int j = 0; j < 6; ++j)
                mma_bf16(tmem + kD2Col, smem_desc(sbase + kOffA2 + 256u * j, 128, 1536),
                         smem_desc(sbase + kOffB2 + 3072u + 256u * j, 128, 1536), i2, 1u);
            if constexpr (Split) {
#pragma unroll
                for (int j = 0; j < 6; ++j)
                    mma_bf16(tmem + kD2Col, smem_desc(sbase + kOffA2lo + 256u * j, 128, 1536),
                             smem_desc(sbase + kOffB2 + 256u * j, 128, 1536), i2, 1u);
            }
            mma_commit(bar2);
        }
        ok = __syncthreads_and(mbar_wait(bar2, phase)) != 0;
        fence_after();
        if (!ok) {
            if (tid == 0 && p.error_flags) atomicOr(p.error_flags, kErrTensorWait);
            break;
        }
        uint32_t r2[4];
        tmem_ld4(lane_base + kD2Col, r2);
        phase ^= 1u;
        if (!live) continue;

        float raw[3] = {__uint_as_float(r2[0]), __uint_as_float(r2[1]), __uint_as_float(r2[2])};
        if (!finite) print_spectral_nonfinite(p.spectral, d, raw);
        if constexpr (Out == 2) { // the spectral integral itself
            p.lin_r[idx] = raw[0];
            p.lin_g[idx] = raw[1];
            p.lin_b[idx] = raw[2];
            continue;
        }
        print_finish(p, blob, raw, d, p.film_dust ? p.film_dust[idx] : 1.0f);
        double rgb[3];
        if constexpr (Out == 1) { // linear output-RGB planes
            const float glare = p.scan_glare ? p.scan_glare[idx] : -1.0f;
            if (!scan_to_linear(p, d, rgb, glare, nullptr)) {
                flag_scan_failure(p);
                rgb[0] = rgb[1] = rgb[2] = 0.0;
            }
            p.lin_r[idx] = (float)rgb[0];
            p.lin_g[idx] = (float)rgb[1];
            p.lin_b[idx] = (float)rgb[2];
            continue;
        }
        const int y = (int)(idx / p.width);
        const int x = (int)(idx - (long long)y * p.width);
        float* dstPix = reinterpret_cast<float*>(p.dst + (long long)y * p.dst_row_bytes) + (long long)x * p.components;
        const float* srcPix =
            p.src ? reinterpret_cast<const float*>(p.src + (long long)y * p.src_row_bytes) + (long long)x * p.components
                  : nullptr;
        if (!scan_to_linear(p, d, rgb, -1.0f, nullptr)) {
            flag_scan_failure(p);
            dstPix[0] = dstPix[1] = dstPix[2] = 0.0f;
            if (p.components == 4) dstPix[3] = srcPix ? srcPix[3] : 1.0f;
            continue;
        }
        encode_output(p, rgb);
        dstPix[0] = (float)rgb[0];
        dstPix[1] = (float)rgb[1];
        dstPix[2] = (float)rgb[2];
        if (p.components == 4) dstPix[3] = srcPix ? srcPix[3] : 1.0f;
    }

    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

template <int Out, bool Split>
cudaError_t launch_tc(const PixelParams& p, cudaStream_t stream) {
    auto* k = print_tc_kernel<Out, Split>;
    // Shared memory sized so that at most four (two for the split form) CTAs share an
    // SM: their TMEM allocations (128 columns each) then always fit the SM's 512.
    size_t smem = off_blob(Split) + (size_t)p.curve_blob_floats * sizeof(float);
    const size_t floor_bytes = Split ? 80 * 1024 : 58 * 1024;
    if (smem < floor_bytes) smem = floor_bytes;
    const int per_sm = Split ? 2 : 4;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (sms <= 0) sms = 148;
    const long long total = (long long)p.width * (long long)p.height;
    const long long tiles = (total + kTcThreads - 1) / kTcThreads;
    const long long cap = (long long)sms * per_sm;
    const int grid = (int)(tiles < cap ? tiles : cap);
    fjb::count_launch();
    k<<<grid, kTcThreads, smem, stream>>>(p);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_print_tensor(const PixelParams& p, PixelStage stage, cudaStream_t stream) {
    const long long total = (long long)p.width * (long long)p.height;
    if (total <= 0) return cudaSuccess;
    if ((p.curve_blob_floats & 3) != 0 || p.spectral.count > kTcLambda || p.spectral.count < 0)
        return cudaErrorInvalidValue;
    const bool split = p.print_form == kPrintTensorSplit;
    switch (stage) {
        case PixelStage::DensityToOutput:
            return split ? launch_tc<0, true>(p, stream) : launch_tc<0, false>(p, stream);
        case PixelStage::DensityToLinearRgb:
            return split ? launch_tc<1, true>(p, stream) : launch_tc<1, false>(p, stream);
        case PixelStage::DensityToPrintRaw:
            return split ? launch_tc<2, true>(p, stream) : launch_tc<2, false>(p, stream);
        default:
            return cudaErrorInvalidValue;
    }
}

} // namespace fjb
