// fjb_print_tc.cu -- the print stage with its 81-wavelength contraction on the
// fifth-generation tensor cores (tcgen05, sm_100a only).
//
// Reference: print_spectral_integrate_device (src/Cuda/JuicerCudaDeviceHelpers.cuh:866-935)
//   D(l) = sum_c d_c eps_c(l) + base(l),  T(l) = 10^-D(l) I_filt(l),  raw_c = sum_l T(l) S_c(l).
// The recipe folds it into nd(l) = -(eps_c, eps_m, eps_y)(l) log2(10), nd3(l) = 0 and
// sens(l) = S(l) I_filt(l) 10^-base(l) (fjb_params.h), so T(l) = 2^(d . nd(l) + nd3(l))
// and raw_c = sum_l T(l) sens_c(l); nd3 is -inf on the padded wavelengths.
//
// One persistent CTA of 128 threads takes tiles of 128 consecutive pixels (one per
// thread, one TMEM lane per pixel):
//   GEMM1  D1[128 x 96] = A1[128 x 16] B1[96 x 16]^T  (M = pixels, N = wavelengths
//          padded 81 -> 96, K = 16). A1 row = (d_hi[3], d_lo[3], d_hi[3], 1, 1, 0...),
//          B1 row = (nd_hi[3], nd_hi[3], nd_lo[3], nd3_hi, nd3_lo, 0...): BF16 hi + lo
//          pairs of both sides, so d . nd + nd3 is carried to about 2^-17 relative
//          (only d_lo nd_lo is dropped), accumulated in FP32 in TMEM.
//   exp2   per pixel and wavelength in FP32 on the MUFU, read from TMEM with
//          tcgen05.ld; T rounded to BF16 (kPrintTensor) or to a BF16 pair hi + lo
//          (kPrintTensorSplit) into shared memory.
//   GEMM2  D2[128 x 16] = T[128 x 96] B2[16 x 96]^T with B2 rows (sens_hi C, M, Y,
//          sens_lo C, M, Y, 0...): six K-steps of 16 (six more for T_lo), FP32
//          accumulate; raw_c = D2[c] + D2[3 + c].
// The tiles are software-pipelined two deep (double-buffered operands and D2): in
// iteration i the CTA turns D1(i) into T(i), issues GEMM2(i) and GEMM1(i + 1) after one
// barrier, prefetches the densities of tile i + 2, then reads raw(i - 1) from TMEM, so
// each MMA runs while the CTA works on another tile. The kernel writes the spectral
// integral planes; the print development, scan and output encoding of each pixel
// follow in the FP32 pixel-chain kernel at full occupancy (fjb_pixel_chain.cu,
// kInPrintRaw), the same device functions as the FP32 form.
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

// shared-memory map, bytes from the (128-aligned) dynamic base; buffers [2] alternate
// between consecutive tiles
constexpr uint32_t kOffA1 = 0;       // 2 x (128 x 16 BF16, 4096 B)
constexpr uint32_t kOffB1 = 8192;    // 96 x 16 BF16 (3072 B)
constexpr uint32_t kOffB2 = 11264;   // 16 x 96 BF16 (3072 B)
constexpr uint32_t kOffA2 = 14336;   // 2 x (128 x 96 BF16 T hi, 24576 B)
constexpr uint32_t kOffA2lo = 63488; // 2 x (128 x 96 BF16 T lo), split form only
__host__ __device__ constexpr uint32_t off_bar(bool split) { return split ? 112640u : 63488u; }
constexpr uint32_t kA1Bytes = 4096, kA2Bytes = 24576;
// TMEM columns: D1 at 0..95 (one buffer: GEMM1(i + 1) is issued only after every thread
// has read D1(i)), D2 of buffer b at 96 + 16 b
constexpr uint32_t kTmemAlloc = 128;
constexpr uint32_t kD2Col = 96;

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

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
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

// A1 row of one pixel (zeros for a dead or non-finite pixel) into buffer `a1`.
__device__ __forceinline__ void write_a1(unsigned char* a1, int tid, const float d[3], bool finite) {
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
    *reinterpret_cast<uint4*>(a1 + kmajor(tid, 0, kTcK1)) = *reinterpret_cast<const uint4*>(a);
    *reinterpret_cast<uint4*>(a1 + kmajor(tid, 8, kTcK1)) = *reinterpret_cast<const uint4*>(a + 8);
}

__device__ __forceinline__ void load_density(const PixelParams& p, long long idx, long long total, float d[3]) {
    if (idx < total) {
        d[0] = __ldg(p.scan_density_c + idx);
        d[1] = __ldg(p.scan_density_m + idx);
        d[2] = __ldg(p.scan_density_y + idx);
    } else {
        d[0] = d[1] = d[2] = 0.0f;
    }
}

__device__ __forceinline__ bool all_finite(const float d[3]) {
    return isfinite(d[0]) && isfinite(d[1]) && isfinite(d[2]);
}

// Spectral integral planes (raw C, M, Y) of the density planes, tile pipeline above.
template <bool Split>
__global__ void __launch_bounds__(kTcThreads, 1) print_raw_tc_kernel(const __grid_constant__ PixelParams p,
                                                                  float* __restrict__ raw_c,
                                                                  float* __restrict__ raw_m,
                                                                  float* __restrict__ raw_y) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const uint32_t sbase = smem_addr(tc_smem);
    uint64_t* bars = reinterpret_cast<uint64_t*>(tc_smem + off_bar(Split)); // bar1[0..1], bar2[0..1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + off_bar(Split) + 32);
    const uint32_t bar1[2] = {smem_addr(bars), smem_addr(bars + 1)};
    const uint32_t bar2[2] = {smem_addr(bars + 2), smem_addr(bars + 3)};

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
    // B2 rows: sens hi C, M, Y, sens lo C, M, Y, zeros; K = wavelength
    for (int e = tid; e < 16 * kTcLambda; e += kTcThreads) {
        const int n = e / kTcLambda, l = e - n * kTcLambda;
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (n < 6 && l < count) {
            __nv_bfloat16 hi, lo;
            split_bf16(p.spectral.sens[l][n % 3], hi, lo);
            v = n < 3 ? hi : lo;
        }
        *reinterpret_cast<__nv_bfloat16*>(tc_smem + kOffB2 + kmajor(n, l, kTcLambda)) = v;
    }
    if (tid == 0) {
        for (int b = 0; b < 4; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + b)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kTmemAlloc)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }

    const long long total = (long long)p.width * (long long)p.height;
    const long long tiles = (total + kTcThreads - 1) / kTcThreads;
    const long long n = tiles > blockIdx.x ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0; // tiles of this CTA
    auto tile_idx = [&](long long j) { return (blockIdx.x + j * (long long)gridDim.x) * kTcThreads + tid; };

    // prologue: A1 of tile 0, densities of tile 1
    float d_cur[3], d_next[3];
    load_density(p, n > 0 ? tile_idx(0) : total, total, d_cur);
    bool fin_cur = tile_idx(0) < total && all_finite(d_cur);
    write_a1(tc_smem + kOffA1, tid, d_cur, fin_cur);
    load_density(p, n > 1 ? tile_idx(1) : total, total, d_next);
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane = (uint32_t)(warp * 32) << 16;
    const uint32_t i1 = idesc_bf16(128, kTcLambda);
    const uint32_t i2 = idesc_bf16(128, 16);
    if (tid == 0 && n > 0) {
        mma_bf16(tmem, smem_desc(sbase + kOffA1, 128, 256), smem_desc(sbase + kOffB1, 128, 256), i1, 0u);
        mma_commit(bar1[0]);
    }

    bool ok = true;
    bool fin_prev = false;
    float d_prev[3] = {0.0f, 0.0f, 0.0f};
    for (long long i = 0; i < n; ++i) {
        const int b = (int)(i & 1);
        const uint32_t parity = (uint32_t)((i >> 1) & 1);
        // 1. T(i) from D1(i) into A2[b]; A1[b^1] for tile i + 1; then GEMM2(i) and GEMM1(i + 1)
        ok = mbar_wait(bar1[b], parity) && ok;
        fence_after();
        if (__all_sync(0xFFFFFFFFu, ok)) {
#pragma unroll
            for (int chunk = 0; chunk < 3; ++chunk) {
                uint32_t r[32];
                tmem_ld32(tmem + lane + (uint32_t)(chunk * 32), r);
                uint32_t hi[16], lo[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    // columns past the 81 wavelengths meet zero spectra: no exponential
                    const int col = chunk * 32 + 2 * j;
                    const float t0 = col < kSpectralSamples ? mufu_exp2(__uint_as_float(r[2 * j])) : 0.0f;
                    const float t1 = col + 1 < kSpectralSamples ? mufu_exp2(__uint_as_float(r[2 * j + 1])) : 0.0f;
                    hi[j] = pack_bf16(t0, t1);
                    if constexpr (Split) {
                        const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&hi[j]);
                        lo[j] = pack_bf16(t0 - __low2float(h), t1 - __high2float(h));
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t off = kmajor(tid, chunk * 32 + q * 8, kTcLambda);
                    *reinterpret_cast<uint4*>(tc_smem + kOffA2 + b * kA2Bytes + off) =
                        make_uint4(hi[4 * q], hi[4 * q + 1], hi[4 * q + 2], hi[4 * q + 3]);
                    if constexpr (Split)
                        *reinterpret_cast<uint4*>(tc_smem + kOffA2lo + b * kA2Bytes + off) =
                            make_uint4(lo[4 * q], lo[4 * q + 1], lo[4 * q + 2], lo[4 * q + 3]);
                }
            }
        }
        const bool fin_next = i + 1 < n && tile_idx(i + 1) < total && all_finite(d_next);
        if (i + 1 < n) write_a1(tc_smem + kOffA1 + (b ^ 1) * kA1Bytes, tid, d_next, fin_next);
        fence_proxy_async();
        fence_before();
        ok = __syncthreads_and(ok) != 0;
        if (!ok) break;
        if (tid == 0) {
            fence_after();
            const uint32_t a2 = sbase + kOffA2 + b * kA2Bytes;
            const uint32_t d2 = tmem + kD2Col + 16 * b;
#pragma unroll
            for (int j = 0; j < 6; ++j)
                mma_bf16(d2, smem_desc(a2 + 256u * j, 128, 1536), smem_desc(sbase + kOffB2 + 256u * j, 128, 1536), i2,
                         j > 0 ? 1u : 0u);
            if constexpr (Split) {
                const uint32_t a2lo = sbase + kOffA2lo + b * kA2Bytes;
#pragma unroll
                for (int j = 0; j < 6; ++j)
                    mma_bf16(d2, smem_desc(a2lo + 256u * j, 128, 1536), smem_desc(sbase + kOffB2 + 256u * j, 128, 1536),
                             i2, 1u);
            }
            mma_commit(bar2[b]);
            if (i + 1 < n) {
                mma_bf16(tmem, smem_desc(sbase + kOffA1 + (b ^ 1) * kA1Bytes, 128, 256),
                         smem_desc(sbase + kOffB1, 128, 256), i1, 0u);
                mma_commit(bar1[b ^ 1]);
            }
        }
        // 2. densities of tile i + 2 in flight while raw(i - 1) is read out
        float d_after[3];
        load_density(p, i + 2 < n ? tile_idx(i + 2) : total, total, d_after);
        // 3. raw(i - 1) from D2(i - 1)
        if (i >= 1) {
            const int pb = b ^ 1;
            bool got = mbar_wait(bar2[pb], (uint32_t)(((i - 1) >> 1) & 1));
            fence_after();
            if (__all_sync(0xFFFFFFFFu, got)) {
                uint32_t r2[8];
                tmem_ld8(tmem + lane + (uint32_t)(kD2Col + 16 * pb), r2);
                const long long idx = tile_idx(i - 1);
                if (idx < total) {
                    float raw[3];
                    for (int c = 0; c < 3; ++c) raw[c] = __uint_as_float(r2[c]) + __uint_as_float(r2[3 + c]);
                    if (!fin_prev) print_spectral_nonfinite(p.spectral, d_prev, raw);
                    raw_c[idx] = raw[0];
                    raw_m[idx] = raw[1];
                    raw_y[idx] = raw[2];
                }
            } else {
                got = false;
            }
            ok = ok && got;
        }
        for (int c = 0; c < 3; ++c) {
            d_prev[c] = d_cur[c];
            d_cur[c] = d_next[c];
            d_next[c] = d_after[c];
        }
        fin_prev = fin_cur;
        fin_cur = fin_next;
    }
    // the last tile's raw
    if (ok && n > 0) {
        const long long i = n - 1;
        const int b = (int)(i & 1);
        bool got = mbar_wait(bar2[b], (uint32_t)((i >> 1) & 1));
        fence_after();
        if (__all_sync(0xFFFFFFFFu, got)) {
            uint32_t r2[8];
            tmem_ld8(tmem + lane + (uint32_t)(kD2Col + 16 * b), r2);
            const long long idx = tile_idx(i);
            if (idx < total) {
                float raw[3];
                for (int c = 0; c < 3; ++c) raw[c] = __uint_as_float(r2[c]) + __uint_as_float(r2[3 + c]);
                if (!fin_prev) print_spectral_nonfinite(p.spectral, d_prev, raw); // tile n - 1 after the shift
                raw_c[idx] = raw[0];
                raw_m[idx] = raw[1];
                raw_y[idx] = raw[2];
            }
        } else {
            got = false;
        }
        ok = got;
    }
    if (!__syncthreads_and(ok) && tid == 0 && p.error_flags) atomicOr(p.error_flags, kErrTensorWait);

    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemAlloc) : "memory");
    }
}

template <bool Split>
cudaError_t launch_raw_tc(const PixelParams& p, float* raw_c, float* raw_m, float* raw_y, cudaStream_t stream) {
    auto* k = print_raw_tc_kernel<Split>;
    // 62 KiB (110 KiB split) of shared memory per CTA: three (two) CTAs share an SM at
    // most, and their TMEM allocations (128 columns each) always fit the SM's 512.
    const size_t smem = off_bar(Split) + 64;
    const int per_sm = Split ? 2 : 3;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (sms <= 0) sms = 148;
    const long long total = (long long)p.width * (long long)p.height;
    const long long tiles = (total + kTcThreads - 1) / kTcThreads;
    const long long cap = (long long)per_sm * sms;
    const int grid = (int)(tiles < cap ? tiles : cap);
    fjb::count_launch();
    k<<<grid, kTcThreads, smem, stream>>>(p, raw_c, raw_m, raw_y);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_print_tensor(const PixelParams& p, PixelStage stage, cudaStream_t stream) {
    const long long total = (long long)p.width * (long long)p.height;
    if (total <= 0) return cudaSuccess;
    if (p.spectral.count > kTcLambda || p.spectral.count < 0) return cudaErrorInvalidValue;
    const bool split = p.print_form == kPrintTensorSplit;
    if (stage == PixelStage::DensityToPrintRaw)
        return split ? launch_raw_tc<true>(p, p.lin_r, p.lin_g, p.lin_b, stream)
                     : launch_raw_tc<false>(p, p.lin_r, p.lin_g, p.lin_b, stream);
    if (stage != PixelStage::DensityToOutput && stage != PixelStage::DensityToLinearRgb) return cudaErrorInvalidValue;
    if (!p.tc_raw) return cudaErrorInvalidValue;
    float* rc = p.tc_raw;
    float* rm = p.tc_raw + total;
    float* ry = p.tc_raw + 2 * total;
    cudaError_t e = split ? launch_raw_tc<true>(p, rc, rm, ry, stream) : launch_raw_tc<false>(p, rc, rm, ry, stream);
    if (e != cudaSuccess) return e;
    PixelParams q = p;
    q.print_raw_c = rc;
    q.print_raw_m = rm;
    q.print_raw_y = ry;
    return launch_pixel_chain(q, stage == PixelStage::DensityToOutput ? PixelStage::RawToOutput
                                                                      : PixelStage::RawToLinearRgb,
                              stream);
}

} // namespace fjb
