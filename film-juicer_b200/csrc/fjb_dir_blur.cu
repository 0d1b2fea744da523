// fjb_dir_blur.cu -- spatial DIR correction diffusion (a7): filtered = sum_k w_k G_k(raw).
//
// Operators restate src/Cuda/Film/JuicerCudaFilmPipeline.cu: FIR with FP64
// accumulation and half-sample reflection (:388-435; taps from the host Gaussian),
// and the FP64 third-order recursion with reflected-boundary start weights and the
// end-block matrix (:478-780), rows left to right then right to left, columns from
// the visual top (last memory row) down, then back up.
//
// B200 schedule. The recursions are block-parallel: a line is cut into segments of
// kDirSeg samples (the segment processed last in a direction is shorter, or absorbs
// a remainder of fewer than 8 samples). A start kernel forms each line's reflected
// start state with parallel dot products; a partial kernel runs every segment (the
// first from the true start state, the others from a zero state) and keeps its exit
// state; a scan kernel turns those into every segment's entry state (x_{j+1} =
// M x_j + Z_j, M the recursion's state map over one segment); the final kernel runs
// each segment again from its entry state. In exact arithmetic this is the sequential recursion; in FP64 it differs
// from it by rounding. Row kernels stage 32 rows x one segment in shared memory so
// global accesses stay coalesced; column kernels give each lane one column and load
// rows ahead of the recursion. The last column pass evaluates every component at each
// pixel and writes the weighted sum once, so the reference's per-component
// read-modify-write accumulation never reaches HBM.
#include <cuda_runtime.h>

#include <type_traits>

#include "fjb_dir.h"
#include "fjb_launches.h"
#include "fjb_lines.cuh"

namespace fjb {

namespace {

constexpr int kLineThreads = 128;
constexpr int kSeg = kDirSeg;
constexpr int kSegMax = kSeg + 8;  // longest segment: a remainder below 8 joins the last one
constexpr int kAhead = 8;          // column kernels: rows loaded ahead of the recursion

__device__ __forceinline__ int reflect_dir(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * n;
    i %= period;
    if (i < 0) i += period;
    return i >= n ? period - 1 - i : i;
}

// One step of the recursion; the newest state enters last so that the loop-carried
// dependency is a single fused multiply-add.
__device__ __forceinline__ double iir_step(const DirComponentDev& c, double x, double s[3]) {
    const double v = fma(c.fb[0], s[0], fma(c.fb[1], s[1], fma(c.fb[2], s[2], c.ff * x)));
    s[2] = s[1];
    s[1] = s[0];
    s[0] = v;
    return v;
}

__host__ __device__ __forceinline__ int seg_count(int n) {
    if (n <= 0) return 0;
    const int full = n / kSeg, rem = n % kSeg;
    const int ns = full + (rem >= 8 ? 1 : 0);
    return ns > 0 ? ns : 1;
}

// forward segment b: [b*kSeg, ...), the last one running to n
__device__ __forceinline__ void fwd_seg(int n, int b, int& lo, int& hi) {
    lo = b * kSeg;
    hi = b == seg_count(n) - 1 ? n : lo + kSeg;
}

// backward segment b (b-th from the end), the last one starting at 0
__device__ __forceinline__ void bwd_seg(int n, int b, int& lo, int& hi) {
    hi = n - b * kSeg;
    lo = b == seg_count(n) - 1 ? 0 : hi - kSeg;
}

__device__ __forceinline__ double* carry_at(const DirBlurParams& p, int ch, int k, int line, int seg) {
    return p.carry + ((((size_t)ch * kDirMaxComponents + k) * p.lines_max + line) * p.segs_max + seg) * 3;
}

// Start record per (channel, component, line): [0..2] the second pass's start state,
// [3..5] the first pass's reflected start state, [6..8] the column end block.
__device__ __forceinline__ double* start_at(const DirBlurParams& p, int ch, int k, int line) {
    return p.start + (((size_t)ch * kDirMaxComponents + k) * p.lines_max + line) * 9;
}

__device__ __forceinline__ void put3(double* d, const double s[3]) {
    d[0] = s[0];
    d[1] = s[1];
    d[2] = s[2];
}

__device__ __forceinline__ void get3(const double* d, double s[3]) {
    s[0] = d[0];
    s[1] = d[1];
    s[2] = d[2];
}

// Entry state of segment seg >= 1, left in the carry slot by the scan kernel.
__device__ __forceinline__ void scan_entry(const DirComponentDev&, const DirBlurParams& p, int ch, int k, int line,
                                           int seg, double s[3]) {
    get3(carry_at(p, ch, k, line, seg), s);
}

enum DirPassKind : int { kRowsFwd = 0, kRowsBwd = 1, kColsA = 2, kColsB = 3 };

// Carry scan of one pass: turns the exit states (segment 0's true, the others from a
// zero state) into every segment's entry state, in place: entry_1 = exit_0,
// entry_{j+1} = M entry_j + Z_j. One thread per (line, component).
__global__ void __launch_bounds__(kLineThreads) dir_scan_kernel(const __grid_constant__ DirBlurParams p, int pass) {
    const int ch = blockIdx.y;
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    const bool rows = pass == kRowsFwd || pass == kRowsBwd;
    if (line >= (rows ? p.height : p.width)) return;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        const int n = pass == kRowsFwd ? p.width : pass == kRowsBwd ? p.width - c.h_tsize : p.height;
        const int ns = seg_count(n);
        if (ns < 2) continue;
        double s[3];
        get3(carry_at(p, ch, k, line, 0), s);
        // exit states are loaded a batch ahead of the dependent chain and the entry
        // stores (the loads cannot pass the stores to the same buffer otherwise)
        constexpr int B = 8;
        double nz[B][3];
        auto load_batch = [&](int j0) {
#pragma unroll
            for (int t = 0; t < B; ++t) {
                const int j = j0 + t;
                if (j < ns - 1) {
                    get3(carry_at(p, ch, k, line, j), nz[t]);
                } else {
                    nz[t][0] = nz[t][1] = nz[t][2] = 0.0; // the last segment keeps no exit state
                }
            }
        };
        load_batch(1);
        for (int j0 = 1; j0 < ns; j0 += B) {
            double z[B][3];
#pragma unroll
            for (int t = 0; t < B; ++t) {
                z[t][0] = nz[t][0];
                z[t][1] = nz[t][1];
                z[t][2] = nz[t][2];
            }
            if (j0 + B < ns) load_batch(j0 + B);
#pragma unroll
            for (int t = 0; t < B; ++t) {
                const int j = j0 + t;
                if (j >= ns) break;
                put3(carry_at(p, ch, k, line, j), s);
                const double a = c.seg[0] * s[0] + c.seg[1] * s[1] + c.seg[2] * s[2] + z[t][0];
                const double b = c.seg[3] * s[0] + c.seg[4] * s[1] + c.seg[5] * s[2] + z[t][1];
                const double d = c.seg[6] * s[0] + c.seg[7] * s[1] + c.seg[8] * s[2] + z[t][2];
                s[0] = a;
                s[1] = b;
                s[2] = d;
            }
        }
    }
}

// End block from the final state: term[r] = last + sum_q T[r][q] (s[ts-1-q] - last).
__device__ __forceinline__ void end_block(const double* T, int ts, const double s[3], double term[3]) {
    const double last = s[0];
    for (int r = 0; r < ts; ++r) {
        double v = last;
        for (int q = 0; q < ts; ++q) v += T[r * ts + q] * (s[ts - 1 - q] - last);
        term[r] = v;
    }
}

__device__ __forceinline__ void load_rows(float (*tile)[kSegMax + 1], const float* src, int W, int row0, int H,
                                          int lo, int len) {
    for (int r = 0; r < 32; ++r) {
        const int y = row0 + r;
        for (int c = threadIdx.x; c < len; c += 32) tile[r][c] = y < H ? src[(size_t)y * W + lo + c] : 0.0f;
    }
    __syncwarp();
}

__device__ __forceinline__ void store_rows(float (*tile)[kSegMax + 1], float* dst, int W, int row0, int H, int lo,
                                           int len) {
    __syncwarp();
    for (int r = 0; r < 32; ++r) {
        const int y = row0 + r;
        if (y >= H) break;
        for (int c = threadIdx.x; c < len; c += 32) dst[(size_t)y * W + lo + c] = tile[r][c];
    }
    __syncwarp();
}

// Row FIR, FP64 accumulation, one thread per pixel.
__global__ void dir_rows_fir_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.width || y >= p.height) return;
    const float* row = p.raw[ch] + (size_t)y * p.width;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpFir) continue;
        double sum = 0.0;
        if (x - c.radius >= 0 && x + c.radius < p.width) {
            for (int o = -c.radius; o <= c.radius; ++o) sum += (double)row[x + o] * (double)c.taps[o + c.radius];
        } else {
            for (int o = -c.radius; o <= c.radius; ++o)
                sum += (double)row[reflect_dir(x + o, p.width)] * (double)c.taps[o + c.radius];
        }
        p.temp[ch][k][(size_t)y * p.width + x] = isfinite(sum) ? (float)sum : 0.0f;
    }
}

// Reflected start states of the rows: anchor + sum_i w_h[i] (x_i - anchor), one warp
// per row, lanes striding the row, FP64 warp reduction.
__global__ void __launch_bounds__(256) dir_row_starts_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.y;
    const int y = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (y >= p.height) return;
    const float* line = p.raw[ch] + (size_t)y * p.width;
    const double anchor = (double)line[0];
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int i = lane; i < c.h_len; i += 32) {
            const double d = (double)line[i] - anchor;
            a0 += c.h_init[i] * d;
            a1 += c.h_init[c.h_len + i] * d;
            a2 += c.h_init[2 * c.h_len + i] * d;
        }
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (lane == 0) {
            double* st = start_at(p, ch, k, y) + 3;
            st[0] = anchor + a0;
            st[1] = anchor + a1;
            st[2] = anchor + a2;
        }
    }
}

// Rows, left to right: exit states (segment 0 from the reflected start).
__global__ void __launch_bounds__(32) dir_rows_partial_fwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    if (seg >= seg_count(W) - 1) return; // the last segment's exit state is never used
    __shared__ float tile[32][kSegMax + 1];
    int lo, hi;
    fwd_seg(W, seg, lo, hi);
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    load_rows(tile, p.raw[ch], W, row0, H, lo, hi - lo);
    if (y >= H) return;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        double s[3] = {0.0, 0.0, 0.0};
        if (seg == 0) get3(start_at(p, ch, k, y) + 3, s);
        for (int x = 0; x < hi - lo; ++x) iir_step(c, (double)tile[threadIdx.x][x], s);
        put3(carry_at(p, ch, k, y, seg), s);
    }
}

// Rows, left to right: values; the last segment also writes the end block and keeps
// the right-to-left start state.
__global__ void __launch_bounds__(32) dir_rows_final_fwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    __shared__ float tile[32][kSegMax + 1];
    int lo, hi;
    fwd_seg(W, seg, lo, hi);
    const int len = hi - lo;
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        load_rows(tile, p.raw[ch], W, row0, H, lo, len);
        if (y < H) {
            double s[3];
            if (seg == 0)
                get3(start_at(p, ch, k, y) + 3, s);
            else
                scan_entry(c, p, ch, k, y, seg, s);
            for (int x = 0; x < len; ++x) tile[threadIdx.x][x] = (float)iir_step(c, (double)tile[threadIdx.x][x], s);
            if (seg == seg_count(W) - 1) {
                const int ts = c.h_tsize;
                double term[3] = {0.0, 0.0, 0.0};
                end_block(c.h_term, ts, s, term);
                for (int r = 0; r < ts; ++r)
                    if (len - ts + r >= 0) tile[threadIdx.x][len - ts + r] = (float)term[r];
                double* st = start_at(p, ch, k, y);
                for (int h = 0; h < 3; ++h) st[h] = h < ts ? term[h] : s[h];
            }
        }
        store_rows(tile, p.temp[ch][k], W, row0, H, lo, len);
    }
}

// Rows, right to left over [0, W - ts): exit states (first segment from the start state).
__global__ void __launch_bounds__(32) dir_rows_partial_bwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    __shared__ float tile[32][kSegMax + 1];
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        const int n = W - c.h_tsize;
        if (n <= 0 || seg >= seg_count(n) - 1) continue;
        int lo, hi;
        bwd_seg(n, seg, lo, hi);
        load_rows(tile, p.temp[ch][k], W, row0, H, lo, hi - lo);
        if (y < H) {
            double s[3] = {0.0, 0.0, 0.0};
            if (seg == 0) get3(start_at(p, ch, k, y), s);
            for (int x = hi - lo - 1; x >= 0; --x) iir_step(c, (double)tile[threadIdx.x][x], s);
            put3(carry_at(p, ch, k, y, seg), s);
        }
        __syncwarp();
    }
}

// Rows, right to left: values in place.
__global__ void __launch_bounds__(32) dir_rows_final_bwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    __shared__ float tile[32][kSegMax + 1];
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        const int n = W - c.h_tsize;
        if (n <= 0 || seg >= seg_count(n)) continue;
        int lo, hi;
        bwd_seg(n, seg, lo, hi);
        load_rows(tile, p.temp[ch][k], W, row0, H, lo, hi - lo);
        if (y < H) {
            double s[3];
            if (seg == 0)
                get3(start_at(p, ch, k, y), s);
            else
                scan_entry(c, p, ch, k, y, seg, s);
            for (int x = hi - lo - 1; x >= 0; --x)
                tile[threadIdx.x][x] = (float)iir_step(c, (double)tile[threadIdx.x][x], s);
        }
        store_rows(tile, p.temp[ch][k], W, row0, H, lo, hi - lo);
    }
}

// Reflected start states of the columns' first pass (from memory row H-1 upward in
// the visual sense): a block of 32 columns x kStartSlices slices of the start window;
// lanes read consecutive columns, slices split the window, shared-memory reduction.
constexpr int kStartSlices = 8;

__global__ void __launch_bounds__(32 * kStartSlices) dir_col_starts_kernel(const __grid_constant__ DirBlurParams p) {
    __shared__ double part[kStartSlices][3][32];
    const int ch = blockIdx.y;
    const int lane = threadIdx.x & 31, slice = threadIdx.x >> 5;
    const int x = blockIdx.x * 32 + lane;
    const int W = p.width, H = p.height;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        double anchor = 0.0;
        if (x < W) {
            const float* T = p.temp[ch][k];
            anchor = (double)T[(size_t)(H - 1) * W + x];
            for (int i = slice; i < c.v_len; i += kStartSlices) {
                const double d = (double)T[(size_t)(H - 1 - i) * W + x] - anchor;
                a0 += c.v_init[i] * d;
                a1 += c.v_init[c.v_len + i] * d;
                a2 += c.v_init[2 * c.v_len + i] * d;
            }
        }
        part[slice][0][lane] = a0;
        part[slice][1][lane] = a1;
        part[slice][2][lane] = a2;
        __syncthreads();
        if (slice == 0 && x < W) {
            double* st = start_at(p, ch, k, x) + 3;
            for (int h = 0; h < 3; ++h) {
                double t = 0.0;
                for (int q = 0; q < kStartSlices; ++q) t += part[q][h][lane];
                st[h] = anchor + t;
            }
        }
        __syncthreads();
    }
}

// Columns, first pass from memory row H-1 down to row 0 over the row-filtered planes:
// exit states (segment 0 from the reflected start).
__global__ void __launch_bounds__(kLineThreads) dir_cols_partial_a_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H) - 1) return;
    int lo, hi;
    bwd_seg(H, seg, lo, hi);
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        const float* T = p.temp[ch][k];
        double s[3] = {0.0, 0.0, 0.0};
        if (seg == 0) get3(start_at(p, ch, k, x) + 3, s);
        for (int y0 = hi - 1; y0 >= lo; y0 -= kAhead) {
            float v[kAhead];
#pragma unroll
            for (int r = 0; r < kAhead; ++r) v[r] = y0 - r >= lo ? T[(size_t)(y0 - r) * W + x] : 0.0f;
#pragma unroll
            for (int r = 0; r < kAhead; ++r)
                if (y0 - r >= lo) iir_step(c, (double)v[r], s);
        }
        put3(carry_at(p, ch, k, x, seg), s);
    }
}

// Columns, first pass: values in place; the segment holding memory row 0 keeps the
// end block and the second pass's start state.
__global__ void __launch_bounds__(kLineThreads) dir_cols_final_a_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H)) return;
    int lo, hi;
    bwd_seg(H, seg, lo, hi);
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        float* T = p.temp[ch][k];
        double s[3];
        if (seg == 0)
            get3(start_at(p, ch, k, x) + 3, s);
        else
            scan_entry(c, p, ch, k, x, seg, s);
        for (int y0 = hi - 1; y0 >= lo; y0 -= kAhead) {
            float v[kAhead];
#pragma unroll
            for (int r = 0; r < kAhead; ++r) v[r] = y0 - r >= lo ? T[(size_t)(y0 - r) * W + x] : 0.0f;
#pragma unroll
            for (int r = 0; r < kAhead; ++r)
                if (y0 - r >= lo) T[(size_t)(y0 - r) * W + x] = (float)iir_step(c, (double)v[r], s);
        }
        if (lo == 0) {
            const int ts = c.v_tsize;
            double term[3] = {0.0, 0.0, 0.0};
            end_block(c.v_term, ts, s, term);
            double* st = start_at(p, ch, k, x);
            for (int h = 0; h < 3; ++h) {
                st[h] = h < ts ? term[h] : s[h];
                st[6 + h] = term[h];
            }
        }
    }
}

// Columns, second pass over memory rows [ts, H): exit states (segment 0 from the
// start state at row ts).
__global__ void __launch_bounds__(kLineThreads) dir_cols_partial_b_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H) - 1) return;
    int lo, hi;
    fwd_seg(H, seg, lo, hi);
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        const float* T = p.temp[ch][k];
        double s[3] = {0.0, 0.0, 0.0};
        int from = lo;
        if (seg == 0) {
            get3(start_at(p, ch, k, x), s);
            from = c.v_tsize;
        }
        for (int y0 = from; y0 < hi; y0 += kAhead) {
            float v[kAhead];
#pragma unroll
            for (int r = 0; r < kAhead; ++r) v[r] = y0 + r < hi ? T[(size_t)(y0 + r) * W + x] : 0.0f;
#pragma unroll
            for (int r = 0; r < kAhead; ++r)
                if (y0 + r < hi) iir_step(c, (double)v[r], s);
        }
        put3(carry_at(p, ch, k, x, seg), s);
    }
}

// Columns, second pass fused with the weighted sum of every component.
__global__ void __launch_bounds__(kLineThreads) dir_cols_final_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H)) return;
    int lo, hi;
    fwd_seg(H, seg, lo, hi);
    double st[kDirMaxComponents][3];
    double term[kDirMaxComponents][3];
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        const double* start = start_at(p, ch, k, x);
        for (int h = 0; h < 3; ++h) term[k][h] = start[6 + h];
        if (seg == 0)
            get3(start, st[k]);
        else
            scan_entry(c, p, ch, k, x, seg, st[k]);
    }
    const float* raw = p.raw[ch];
    float* dst = p.filtered[ch];
    for (int y = lo; y < hi; ++y) {
        const size_t idx = (size_t)y * W + x;
        float acc = 0.0f;
        for (int k = 0; k < p.count; ++k) {
            const DirComponentDev& c = p.comp[k];
            float blurred;
            if (c.op == kDirOpIdentity) {
                blurred = raw[idx];
            } else if (c.op == kDirOpFir) {
                const float* T = p.temp[ch][k];
                double sum = 0.0;
                if (y - c.radius >= 0 && y + c.radius < H) {
                    for (int o = -c.radius; o <= c.radius; ++o)
                        sum += (double)T[(size_t)(y + o) * W + x] * (double)c.taps[o + c.radius];
                } else {
                    for (int o = -c.radius; o <= c.radius; ++o)
                        sum += (double)T[(size_t)reflect_dir(y + o, H) * W + x] * (double)c.taps[o + c.radius];
                }
                blurred = isfinite(sum) ? (float)sum : 0.0f;
            } else {
                // memory row y is visual row H-1-y; the end block covers memory rows [0, ts)
                const int ts = c.v_tsize;
                if (y < ts)
                    blurred = (float)term[k][ts - 1 - y];
                else
                    blurred = (float)iir_step(c, (double)p.temp[ch][k][idx], st[k]);
            }
            const float weighted = blurred * c.weight;
            acc = k == 0 ? weighted : acc + weighted;
        }
        dst[idx] = acc;
    }
}

// ---------------------------------------------------------------------------
// Shared-memory form, used when whole lines fit on chip (the usual case): a CTA
// holds kRowsPerCta full rows, or a kStripCols-wide strip of full columns, and runs
// the block-parallel recursion of fjb_lines.cuh on them (reflected starts as
// segment-wise partial dot products summed in segment order, the end block from the
// last state), so each component costs one read and one write of the plane per pass.
// ---------------------------------------------------------------------------
constexpr int kRowsPerCta = 4;
constexpr int kStripCols = 8;
// CTA sizes (threads, resident CTAs per SM) that bound registers so shared memory,
// not registers, sets the occupancy
constexpr int kRowsThreads = 256, kRowsBlocks = 3;
constexpr int kColsThreads = 320, kColsBlocks = 2;
constexpr size_t kSmemLimit = 200 * 1024;
static_assert(kDirSeg == lines::kLineSeg, "segment maps are built for the line segment length");

// One recursive component with its coefficients held in registers: the reference's
// FP64 direct form (state y[n-1], y[n-2], y[n-3]).
struct DirStep {
    using Real = double;
    double ff, fb0, fb1, fb2;
    const double* seg;
    const double* seg4;
    __device__ explicit DirStep(const DirComponentDev& c)
        : ff(c.ff), fb0(c.fb[0]), fb1(c.fb[1]), fb2(c.fb[2]), seg(c.seg), seg4(c.seg4) {}
    __device__ __forceinline__ double step(float x, double s[3]) const {
        const double v = fma(fb0, s[0], fma(fb1, s[1], fma(fb2, s[2], ff * (double)x)));
        s[2] = s[1];
        s[1] = s[0];
        s[0] = v;
        return v;
    }
    __device__ __forceinline__ const double* map() const { return seg; }
    __device__ __forceinline__ const double* map4() const { return seg4; }
    __device__ __forceinline__ void from_direct(double*) const {}
    __device__ __forceinline__ void to_direct(const double* s, double d[3]) const {
        d[0] = s[0];
        d[1] = s[1];
        d[2] = s[2];
    }
};

// The same recursion in its factored FP32 form (state u, y, v: first-order output,
// output, last output difference; factor_recursion in fjb_dir_host.cpp). The reflected
// starts and the end block stay FP64 in the direct basis and are mapped at the ends of
// each pass.
struct DirStepF {
    using Real = float;
    float c0, c1, c2;
    const double* seg;
    const double* seg4;
    const double* to_fac;
    const double* from_fac;
    __device__ explicit DirStepF(const DirComponentDev& c)
        : c0(c.fac[0]), c1(c.fac[1]), c2(c.fac[2]), seg(c.seg_f), seg4(c.seg4_f), to_fac(c.to_fac),
          from_fac(c.from_fac) {}
    __device__ __forceinline__ float step(float x, float s[3]) const {
        s[0] = fmaf(c0, x - s[0], s[0]);
        s[2] = fmaf(c2, s[2], c1 * (s[0] - s[1]));
        s[1] += s[2];
        return s[1];
    }
    __device__ __forceinline__ const double* map() const { return seg; }
    __device__ __forceinline__ const double* map4() const { return seg4; }
    __device__ __forceinline__ void from_direct(double s[3]) const {
        const double* T = to_fac;
        const double o0 = T[0] * s[0] + T[1] * s[1] + T[2] * s[2];
        const double o1 = T[3] * s[0] + T[4] * s[1] + T[5] * s[2];
        const double o2 = T[6] * s[0] + T[7] * s[1] + T[8] * s[2];
        s[0] = o0;
        s[1] = o1;
        s[2] = o2;
    }
    __device__ __forceinline__ void to_direct(const float* s, double d[3]) const {
        const double* T = from_fac;
        for (int r = 0; r < 3; ++r) d[r] = T[3 * r] * (double)s[0] + T[3 * r + 1] * (double)s[1] + T[3 * r + 2] * (double)s[2];
    }
};

// Direct-form starts of L lines (doubles in `entry`) to the step's state, in place
// (Step::Real). Ends with a barrier.
template <typename Step>
__device__ void starts_to_state(const Step& op, double* entry, int L) {
    using R = typename Step::Real;
    double s[3] = {0.0, 0.0, 0.0};
    const int line = threadIdx.x;
    if (line < L) {
        for (int h = 0; h < 3; ++h) s[h] = entry[line * 3 + h];
        op.from_direct(s);
    }
    __syncthreads();
    if (line < L) {
        R* e = reinterpret_cast<R*>(entry);
        for (int h = 0; h < 3; ++h) e[line * 3 + h] = (R)s[h];
    }
    __syncthreads();
}

__host__ __device__ inline size_t carry_doubles(int L, int n) { return (size_t)L * lines::scan_chunks(lines::segs(n)) * 3; }

// Exit states of the pieces (L x segs x 3), also the reduction scratch of the
// reflected starts (warps x ceil(L / 4) x 12) for blocks of up to `threads` threads.
__host__ __device__ inline size_t exits_doubles(int L, int n, int threads) {
    const size_t e = (size_t)L * lines::segs(n) * 3, r = (size_t)(threads / 32) * ((L + 3) / 4) * 12;
    return e > r ? e : r;
}

// Nine consecutive outputs per thread in the FIR components (odd, so that the warp's
// threads, nine samples apart, fall in distinct shared-memory banks).
constexpr int kFirRun = 9;
constexpr int kFirWindowMaxRadius = 9;

// Doubles ahead of the rows in the rows kernel: the recursion's exits, entry, last and
// carry arrays, or, for the FIR components, a per-warp staging area of 32 x kFirRun
// floats through which the outputs go out coalesced.
__host__ __device__ inline size_t rows_prefix_doubles(int W) {
    const size_t scan =
        exits_doubles(kRowsPerCta, W, kRowsThreads) + (size_t)kRowsPerCta * 6 + carry_doubles(kRowsPerCta, W);
    const size_t stage = (size_t)(kRowsThreads / 32) * 32 * kFirRun / 2;
    return scan > stage ? scan : stage;
}

size_t rows_smem_bytes(int W) {
    return (size_t)kRowsPerCta * lines::padded(W) * sizeof(float) + rows_prefix_doubles(W) * sizeof(double);
}

size_t cols_smem_bytes(int H) {
    return (size_t)kStripCols * lines::padded(H) * sizeof(float) +
           (exits_doubles(kStripCols, H, kColsThreads) + (size_t)kStripCols * 6 + carry_doubles(kStripCols, H)) *
               sizeof(double);
}

// ---------------------------------------------------------------------------
// FIR components on lines staged densely in shared memory: a thread computes nine
// consecutive outputs from a register window, converting each input to FP64 once
// (instead of once per tap); the taps are summed in order, as the direct loop does.
// Gaussian taps are symmetric, so half of them (as doubles) stay in registers.
// ---------------------------------------------------------------------------
template <int RAD, typename Get, typename Put>
__device__ __forceinline__ void fir_run(const double (&t)[RAD + 1], int p0, int n, Get get, Put put) {
    // streamed over the window: input i adds its term to every output it reaches, in
    // increasing tap order per output; output j is complete (and handed to `put`) once
    // input j + 2 RAD is in
    double sum[kFirRun];
#pragma unroll
    for (int j = 0; j < kFirRun; ++j) sum[j] = 0.0;
#pragma unroll
    for (int i = 0; i < kFirRun + 2 * RAD; ++i) {
        int q = p0 - RAD + i;
        q = (unsigned)q < (unsigned)n ? q : reflect_dir(q, n);
        const double v = (double)get(q);
#pragma unroll
        for (int j = 0; j < kFirRun; ++j) {
            const int o = i - j;
            if (o >= 0 && o <= 2 * RAD) sum[j] += v * t[o <= RAD ? o : 2 * RAD - o];
        }
        if (i >= 2 * RAD) put(i - 2 * RAD, isfinite(sum[i - 2 * RAD]) ? (float)sum[i - 2 * RAD] : 0.0f);
    }
}

template <int RAD>
__device__ __forceinline__ void fir_load_taps(const float* taps, double (&t)[RAD + 1]) {
#pragma unroll
    for (int o = 0; o <= RAD; ++o) t[o] = (double)__ldg(taps + o);
}

// Rows [row0, row0 + L) of `buf` (dense, W floats per row) into plane T. Each warp
// takes 32 consecutive runs at a time and writes them out through its staging area.
template <int RAD>
__device__ void fir_rows(const DirComponentDev& c, const float* buf, int L, int W, int row0, float* T, float* stage) {
    double t[RAD + 1];
    fir_load_taps<RAD>(c.taps, t);
    const int nb = (W + kFirRun - 1) / kFirRun;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    float* st = stage + warp * 32 * kFirRun;
    for (int base = warp * 32; base < L * nb; base += warps * 32) {
        const int task = base + lane;
        if (task < L * nb) {
            const int r = task / nb, p0 = (task - r * nb) * kFirRun;
            const float* row = buf + (size_t)r * W;
            fir_run<RAD>(t, p0, W, [&](int q) { return row[q]; }, [&](int j, float v) { st[lane * kFirRun + j] = v; });
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kFirRun; ++i) {
            const int e = i * 32 + lane;
            const int tk = base + e / kFirRun;
            if (tk < L * nb) {
                const int r = tk / nb, x = (tk - r * nb) * kFirRun + e % kFirRun;
                if (x < W) T[(size_t)(row0 + r) * W + x] = st[e];
            }
        }
        __syncwarp();
    }
}

// Columns of an 8-wide dense strip (element (y, c) at y * 8 + c): weighted and summed
// into the running sum as the component epilogue does.
template <int RAD>
__device__ void fir_cols(const DirComponentDev& c, const float* work, int H, int W, int x0, int k, const float* acc_in,
                         float* acc_out) {
    double t[RAD + 1];
    fir_load_taps<RAD>(c.taps, t);
    const int nrb = (H + kFirRun - 1) / kFirRun;
    for (int task = threadIdx.x; task < 8 * nrb; task += blockDim.x) {
        const int cc = task & 7, p0 = (task >> 3) * kFirRun;
        fir_run<RAD>(t, p0, H, [&](int q) { return work[q * 8 + cc]; }, [&](int j, float blurred) {
            const int y = p0 + j;
            if (y < H) {
                const size_t o = (size_t)y * W + x0 + cc;
                const float weighted = blurred * c.weight;
                acc_out[o] = k == 0 ? weighted : acc_in[o] + weighted;
            }
        });
    }
}

template <typename F>
__device__ __forceinline__ void with_radius(int rad, F f) {
    switch (rad) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 3: f(std::integral_constant<int, 3>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 5: f(std::integral_constant<int, 5>{}); break;
        case 6: f(std::integral_constant<int, 6>{}); break;
        case 7: f(std::integral_constant<int, 7>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        default: f(std::integral_constant<int, 9>{}); break;
    }
}

// Reflected start of each line: anchor + sum_i w_h[i] (x_i - anchor) over the first
// `len` samples in processing order (i counts from the first sample processed). The
// sums run sample-major: a thread takes samples i (strided by the block) for a group of
// four lines, so each weight is read once per group; partial sums are reduced across
// each warp (fixed butterfly order) and then across warps in warp order, in FP64.
// `red` is scratch of (blockDim / 32) x ceil(L / 4) x 12 doubles.
template <int ES, bool kForward, typename Buf>
__device__ void reflected_starts(Buf buf, int L, int n, const double* w, int len, double* red, double* entry) {
    constexpr int G = 4;
    const int groups = (L + G - 1) / G; // 1 or 2: lanes of equal parity share a group when 2
    const int grp = threadIdx.x % groups;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int first = kForward ? 0 : n - 1;
    double anchor[G], acc[G][3];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int line = grp * G + g;
        anchor[g] = line < L ? (double)buf(line)[lines::at(first) * ES] : 0.0;
        acc[g][0] = acc[g][1] = acc[g][2] = 0.0;
    }
    const int stride = blockDim.x / groups;
    for (int i = threadIdx.x / groups; i < len; i += stride) {
        const int idx = lines::at(kForward ? i : n - 1 - i) * ES;
        const double w0 = w[i], w1 = w[len + i], w2 = w[2 * len + i];
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int line = grp * G + g;
            if (line < L) {
                const double d = (double)buf(line)[idx] - anchor[g];
                acc[g][0] += w0 * d;
                acc[g][1] += w1 * d;
                acc[g][2] += w2 * d;
            }
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int r = 0; r < 3; ++r)
            for (int o = 16; o >= groups; o >>= 1) acc[g][r] += __shfl_xor_sync(0xffffffffu, acc[g][r], o);
    if (lane < groups) {
        double* q = red + ((size_t)warp * groups + lane) * (G * 3);
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int r = 0; r < 3; ++r) q[g * 3 + r] = acc[g][r];
    }
    __syncthreads();
    const int nwarps = blockDim.x >> 5;
    for (int t = threadIdx.x; t < L * 3; t += blockDim.x) {
        const int line = t / 3, r = t - line * 3;
        const int g = line / G, k = line - g * G;
        double sum = 0.0;
        for (int wi = 0; wi < nwarps; ++wi) sum += red[((size_t)wi * groups + g) * (G * 3) + k * 3 + r];
        entry[t] = (double)buf(line)[lines::at(first) * ES] + sum;
    }
    __syncthreads();
}

// One recursive component over the L rows of the CTA, in place: the reflected start,
// left to right, the end block at the last ts samples, right to left from it.
template <typename Step, typename Buf>
__device__ void yvv_rows(const DirComponentDev& c, Buf line, int L, int W, double* exits, double* entry,
                         double* last, double* carry) {
    using R = typename Step::Real;
    const Step op(c);
    reflected_starts<1, true>(line, L, W, c.h_init, c.h_len, exits, entry);
    starts_to_state(op, entry, L);
    lines::run_direction<1, true>(op, line, L, 0, W, reinterpret_cast<R*>(entry), reinterpret_cast<R*>(exits), carry,
                                  reinterpret_cast<R*>(last), false);
    const int ts = c.h_tsize;
    for (int r = threadIdx.x; r < L; r += blockDim.x) {
        double d[3], term[3] = {0.0, 0.0, 0.0};
        op.to_direct(reinterpret_cast<R*>(last) + r * 3, d);
        end_block(c.h_term, ts, d, term);
        for (int q = 0; q < ts; ++q)
            if (W - ts + q >= 0) line(r)[lines::at(W - ts + q)] = (float)term[q];
        for (int h = 0; h < 3; ++h) entry[r * 3 + h] = h < ts ? term[h] : d[h];
    }
    __syncthreads();
    starts_to_state(op, entry, L);
    if (W - ts > 0)
        lines::run_direction<1, false>(op, line, L, 0, W - ts, reinterpret_cast<R*>(entry), reinterpret_cast<R*>(exits),
                                       carry, (R*)nullptr, false);
}

// One recursive component over the kStripCols columns of the CTA: from the visual top
// (memory row H-1) down with the reflected start, the end block at rows [0, ts) (kept
// in `terms`), back up from row ts.
template <typename Step, typename Buf>
__device__ void yvv_cols(const DirComponentDev& c, Buf column, int H, double* exits, double* entry, double* last,
                         double* carry, double (*terms)[3]) {
    using R = typename Step::Real;
    const Step op(c);
    const int ts = c.v_tsize;
    reflected_starts<kStripCols, false>(column, kStripCols, H, c.v_init, c.v_len, exits, entry);
    starts_to_state(op, entry, kStripCols);
    lines::run_direction<kStripCols, false>(op, column, kStripCols, 0, H, reinterpret_cast<R*>(entry),
                                            reinterpret_cast<R*>(exits), carry, reinterpret_cast<R*>(last), true);
    for (int cc = threadIdx.x; cc < kStripCols; cc += blockDim.x) {
        double d[3], term[3] = {0.0, 0.0, 0.0};
        op.to_direct(reinterpret_cast<R*>(last) + cc * 3, d);
        end_block(c.v_term, ts, d, term);
        for (int h = 0; h < 3; ++h) {
            terms[cc][h] = term[h];
            entry[cc * 3 + h] = h < ts ? term[h] : d[h];
        }
    }
    __syncthreads();
    starts_to_state(op, entry, kStripCols);
    if (H - ts > 0)
        lines::run_direction<kStripCols, true>(op, column, kStripCols, ts, H - ts, reinterpret_cast<R*>(entry),
                                               reinterpret_cast<R*>(exits), carry, (R*)nullptr, true);
}

// Rows: every component into its row-filtered plane (recursive: left to right, end
// block, right to left; FIR: reflect taps in FP64).
__global__ void __launch_bounds__(kRowsThreads, kRowsBlocks) dir_rows_smem_kernel(const __grid_constant__ DirBlurParams p) {
    extern __shared__ __align__(16) unsigned char dsm[];
    const int ch = blockIdx.y;
    const int W = p.width, H = p.height;
    const int row0 = blockIdx.x * kRowsPerCta;
    const int L = min(kRowsPerCta, H - row0);
    const int pw = lines::padded(W);
    double* exits = reinterpret_cast<double*>(dsm);
    double* entry = exits + exits_doubles(kRowsPerCta, W, kRowsThreads);
    double* last = entry + (size_t)kRowsPerCta * 3;
    double* carry = last + (size_t)kRowsPerCta * 3;
    float* buf = reinterpret_cast<float*>(exits + rows_prefix_doubles(W));
    auto line = [&](int r) { return buf + (size_t)r * pw; };
    const float* raw = p.raw[ch];
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op == kDirOpFir) {
            // reflect-boundary taps in FP64 over the densely staged rows
            lines::load_rows_dense(buf, raw, W, row0, L, W);
            const int rad = c.radius;
            if (c.symmetric_taps && rad >= 1 && rad <= kFirWindowMaxRadius) {
                float* T = p.temp[ch][k];
                float* stage = reinterpret_cast<float*>(exits);
                with_radius(rad, [&](auto R) { fir_rows<decltype(R)::value>(c, buf, L, W, row0, T, stage); });
                __syncthreads();
                continue;
            }
            for (int r = 0; r < L; ++r) {
                const float* row = buf + (size_t)r * W;
                float* out = p.temp[ch][k] + (size_t)(row0 + r) * W;
                for (int x = threadIdx.x; x < W; x += blockDim.x) {
                    double sum = 0.0;
                    if (x - rad >= 0 && x + rad < W)
                        for (int o = -rad; o <= rad; ++o) sum += (double)row[x + o] * (double)c.taps[o + rad];
                    else
                        for (int o = -rad; o <= rad; ++o)
                            sum += (double)row[reflect_dir(x + o, W)] * (double)c.taps[o + rad];
                    out[x] = isfinite(sum) ? (float)sum : 0.0f;
                }
            }
            __syncthreads();
            continue;
        }
        if (c.op != kDirOpYvv) continue;
        lines::load_rows(buf, raw, W, row0, L, W);
        if (c.factored)
            yvv_rows<DirStepF>(c, line, L, W, exits, entry, last, carry);
        else
            yvv_rows<DirStep>(c, line, L, W, exits, entry, last, carry);
        lines::store_rows(buf, p.temp[ch][k], row0, L, W);
    }
}

// Columns of a kStripCols-wide strip: every component in order (recursive: from the
// visual top, memory row H-1, down to row 0 with the reflected start, end block at
// rows [0, ts), back up from row ts; FIR: reflect taps in FP64; identity), weighted
// and summed as the reference accumulates them, into the filtered plane. The running
// sum is parked in the strip of the row-filtered plane this CTA has just consumed (it
// stays in L2), which keeps shared memory to one strip.
__global__ void __launch_bounds__(kColsThreads, kColsBlocks) dir_cols_smem_kernel(const __grid_constant__ DirBlurParams p) {
    extern __shared__ __align__(16) unsigned char dsm[];
    const int ch = blockIdx.y;
    const int W = p.width, H = p.height;
    const int x0 = blockIdx.x * kStripCols;
    const int C = min(kStripCols, W - x0);
    double* exits = reinterpret_cast<double*>(dsm);
    double* entry = exits + exits_doubles(kStripCols, H, kColsThreads);
    double* last = entry + (size_t)kStripCols * 3;
    double* carry = last + (size_t)kStripCols * 3;
    float* work = reinterpret_cast<float*>(carry + carry_doubles(kStripCols, H));
    auto column = [&](int cc) { return work + cc; };
    const float* raw = p.raw[ch];
    __shared__ double terms[kStripCols][3];
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        const bool final_comp = k == p.count - 1;
        const float* acc_in = k > 0 ? p.temp[ch][k - 1] : nullptr;
        float* acc_out = final_comp ? p.filtered[ch] : p.temp[ch][k];
        const bool reads_raw = c.op == kDirOpIdentity;
        // full strips on 16-byte aligned planes move four columns per access
        const bool vec = C == kStripCols && W % 4 == 0 && lines::aligned16(raw) && lines::aligned16(acc_out) &&
                         (reads_raw || lines::aligned16(p.temp[ch][k])) && (!acc_in || lines::aligned16(acc_in));
        const bool dense_fir = vec && c.op == kDirOpFir;
        if (dense_fir)
            lines::load_strip8_dense(work, p.temp[ch][k], W, H, x0);
        else if (!reads_raw)
            lines::load_strip8(work, p.temp[ch][k], W, H, x0, C);
        const int ts = c.v_tsize;
        if (c.op == kDirOpYvv) {
            if (c.factored)
                yvv_cols<DirStepF>(c, column, H, exits, entry, last, carry, terms);
            else
                yvv_cols<DirStep>(c, column, H, exits, entry, last, carry, terms);
        }
        auto accumulate = [&](float blurred, float a) {
            const float weighted = blurred * c.weight;
            return k == 0 ? weighted : a + weighted;
        };
        if (dense_fir && c.symmetric_taps && c.radius >= 1 && c.radius <= kFirWindowMaxRadius) {
            with_radius(c.radius,
                        [&](auto R) { fir_cols<decltype(R)::value>(c, work, H, W, x0, k, acc_in, acc_out); });
        } else if (vec) {
            // thread -> (row, half strip); global reads go kBatch rows at a time
            constexpr int kBatch = 4;
            const int h = threadIdx.x & 1, ys = blockDim.x >> 1;
            for (int y0 = threadIdx.x >> 1; y0 < H; y0 += kBatch * ys) {
                float4 rawv[kBatch], accv[kBatch];
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ys;
                    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    rawv[b] = reads_raw && y < H ? *reinterpret_cast<const float4*>(raw + (size_t)y * W + x0 + 4 * h) : z;
                    accv[b] = acc_in && y < H ? *reinterpret_cast<const float4*>(acc_in + (size_t)y * W + x0 + 4 * h) : z;
                }
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ys;
                    if (y >= H) continue;
                    float4 v;
                    if (reads_raw) {
                        v = rawv[b];
                    } else if (c.op == kDirOpFir) {
                        // four columns per tap from the dense strip, each summed in FP64
                        double sx = 0.0, sy = 0.0, sz = 0.0, sw = 0.0;
                        for (int o = -c.radius; o <= c.radius; ++o) {
                            const float4 t = *reinterpret_cast<const float4*>(work + reflect_dir(y + o, H) * 8 + 4 * h);
                            const double wt = (double)c.taps[o + c.radius];
                            sx += (double)t.x * wt;
                            sy += (double)t.y * wt;
                            sz += (double)t.z * wt;
                            sw += (double)t.w * wt;
                        }
                        v = make_float4(isfinite(sx) ? (float)sx : 0.0f, isfinite(sy) ? (float)sy : 0.0f,
                                        isfinite(sz) ? (float)sz : 0.0f, isfinite(sw) ? (float)sw : 0.0f);
                    } else if (y < ts) {
                        const int cc = 4 * h;
                        v = make_float4((float)terms[cc][ts - 1 - y], (float)terms[cc + 1][ts - 1 - y],
                                        (float)terms[cc + 2][ts - 1 - y], (float)terms[cc + 3][ts - 1 - y]);
                    } else {
                        v = *reinterpret_cast<const float4*>(work + lines::at(y) * 8 + 4 * h);
                    }
                    const float4 a = accv[b];
                    *reinterpret_cast<float4*>(acc_out + (size_t)y * W + x0 + 4 * h) =
                        make_float4(accumulate(v.x, a.x), accumulate(v.y, a.y), accumulate(v.z, a.z),
                                    accumulate(v.w, a.w));
                }
            }
        } else {
            // one column per thread (the block size is a multiple of kStripCols)
            constexpr int kBatch = 8;
            const int cc = threadIdx.x % kStripCols, ystep = blockDim.x / kStripCols;
            for (int y0 = threadIdx.x / kStripCols; y0 < H; y0 += kBatch * ystep) {
                float rawv[kBatch], accv[kBatch];
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ystep;
                    const bool in = y < H && cc < C;
                    rawv[b] = reads_raw && in ? raw[(size_t)y * W + x0 + cc] : 0.0f;
                    accv[b] = acc_in && in ? acc_in[(size_t)y * W + x0 + cc] : 0.0f;
                }
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ystep;
                    if (y >= H || cc >= C) continue;
                    float blurred;
                    if (reads_raw) {
                        blurred = rawv[b];
                    } else if (c.op == kDirOpFir) {
                        double sum = 0.0;
                        for (int o = -c.radius; o <= c.radius; ++o)
                            sum += (double)work[lines::at(reflect_dir(y + o, H)) * kStripCols + cc] *
                                   (double)c.taps[o + c.radius];
                        blurred = isfinite(sum) ? (float)sum : 0.0f;
                    } else {
                        blurred = y < ts ? (float)terms[cc][ts - 1 - y] : work[lines::at(y) * kStripCols + cc];
                    }
                    acc_out[(size_t)y * W + x0 + cc] = accumulate(blurred, accv[b]);
                }
            }
        }
        __syncthreads();
    }
}

} // namespace

int dir_segments(int n) { return seg_count(n); }

cudaError_t launch_dir_blur(const DirBlurParams& p, cudaStream_t stream) {
    if (p.width <= 0 || p.height <= 0 || p.count <= 0) return cudaSuccess;
    bool fir = false, iir = false;
    for (int k = 0; k < p.count; ++k) {
        fir |= p.comp[k].op == kDirOpFir;
        iir |= p.comp[k].op == kDirOpYvv;
    }
    const int W = p.width, H = p.height;
    const dim3 rows_grid((H + 31) / 32, seg_count(W), 3);
    const dim3 cols_grid((W + kLineThreads - 1) / kLineThreads, seg_count(H), 3);
    cudaError_t e = cudaSuccess;
    // whole rows / column strips in shared memory when they fit, else the global form
    const size_t rs = rows_smem_bytes(W), cs = cols_smem_bytes(H);
    const bool rows_on_chip = rs <= kSmemLimit, cols_on_chip = cs <= kSmemLimit;
    if (fir && !rows_on_chip) {
        const dim3 block(32, 8);
        fjb::count_launch();
        dir_rows_fir_kernel<<<dim3((W + 31) / 32, (H + 7) / 8, 3), block, 0, stream>>>(p);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if ((iir || fir) && rows_on_chip) {
        if ((e = cudaFuncSetAttribute(dir_rows_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rs)) !=
            cudaSuccess)
            return e;
        fjb::count_launch();
        dir_rows_smem_kernel<<<dim3((H + kRowsPerCta - 1) / kRowsPerCta, 3), lines::line_threads(kRowsPerCta, W, kRowsThreads), rs,
                               stream>>>(p);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else if (iir) {
        fjb::count_launch();
        dir_row_starts_kernel<<<dim3((H + 7) / 8, 3), 256, 0, stream>>>(p);
        const dim3 row_lines((H + kLineThreads - 1) / kLineThreads, 3);
        fjb::count_launch();
        dir_rows_partial_fwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        fjb::count_launch();
        dir_scan_kernel<<<row_lines, kLineThreads, 0, stream>>>(p, kRowsFwd);
        fjb::count_launch();
        dir_rows_final_fwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        fjb::count_launch();
        dir_rows_partial_bwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        fjb::count_launch();
        dir_scan_kernel<<<row_lines, kLineThreads, 0, stream>>>(p, kRowsBwd);
        fjb::count_launch();
        dir_rows_final_bwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (cols_on_chip) {
        if ((e = cudaFuncSetAttribute(dir_cols_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs)) !=
            cudaSuccess)
            return e;
        fjb::count_launch();
        dir_cols_smem_kernel<<<dim3((W + kStripCols - 1) / kStripCols, 3), lines::line_threads(kStripCols, H, kColsThreads), cs,
                               stream>>>(p);
        return cudaGetLastError();
    }
    if (iir) {
        const dim3 col_lines((W + kLineThreads - 1) / kLineThreads, 3);
        fjb::count_launch();
        dir_col_starts_kernel<<<dim3((W + 31) / 32, 3), 32 * kStartSlices, 0, stream>>>(p);
        fjb::count_launch();
        dir_cols_partial_a_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
        fjb::count_launch();
        dir_scan_kernel<<<col_lines, kLineThreads, 0, stream>>>(p, kColsA);
        fjb::count_launch();
        dir_cols_final_a_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
        fjb::count_launch();
        dir_cols_partial_b_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
        fjb::count_launch();
        dir_scan_kernel<<<col_lines, kLineThreads, 0, stream>>>(p, kColsB);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    fjb::count_launch();
    dir_cols_final_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
    return cudaGetLastError();
}

} // namespace fjb
