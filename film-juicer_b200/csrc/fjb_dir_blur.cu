// fjb_dir_blur.cu -- spatial DIR correction diffusion (a7): filtered = sum_k w_k G_k(raw).
//
// Operators restate src/Cuda/Film/JuicerCudaFilmPipeline.cu: FIR with FP64
// accumulation and half-sample reflection (:388-435; taps from the host Gaussian),
// and the FP64 third-order recursion with reflected-boundary start weights and the
// end-block matrix (:478-780), rows left to right then right to left, columns from
// the visual top (last memory row) down, then back up.
//
// B200 schedule: all components of all three correction planes are computed in two
// launches plus one fused column launch: row FIR (thread per pixel, grid.z =
// channel), row recursion (thread per row, grid.y = channel), and a column kernel
// (thread per column, grid.y = channel) that runs every recursive component's
// first column pass in place and then one final sweep that evaluates all components
// at each pixel and writes the weighted sum once, so the reference's per-component
// read-modify-write accumulation never reaches HBM.
#include <cuda_runtime.h>

#include "fjb_dir.h"
#include "fjb_launches.h"

namespace fjb {

namespace {

constexpr int kLineThreads = 128;

__device__ __forceinline__ int reflect_dir(int i, int n) {
    if (n <= 1) return 0;
    const int period = 2 * n;
    i %= period;
    if (i < 0) i += period;
    return i >= n ? period - 1 - i : i;
}

__device__ __forceinline__ double iir_step(const DirComponentDev& c, double x, double s[3]) {
    const double v = c.ff * x + c.fb[0] * s[0] + c.fb[1] * s[1] + c.fb[2] * s[2];
    s[2] = s[1];
    s[1] = s[0];
    s[0] = v;
    return v;
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
        for (int o = -c.radius; o <= c.radius; ++o)
            sum += (double)row[reflect_dir(x + o, p.width)] * (double)c.taps[o + c.radius];
        p.temp[ch][k][(size_t)y * p.width + x] = isfinite(sum) ? (float)sum : 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Recursive components, block-parallel in FP64. Lines are cut into segments of
// kDirSeg samples (the segment processed last in a direction absorbs the remainder).
// The partial kernels run every segment but the first from a zero state and keep its
// exit state; the first segment starts from the line's true start state (reflected
// start weights, or the end block) and keeps its true exit state. The final kernels
// rebuild each segment's entry state from those (x_{j+1} = M x_j + Z_j, M the
// recursion's state map over one segment) and run the segment again. In exact
// arithmetic this is the sequential recursion; in FP64 it differs from it by
// rounding. Row kernels stage 32 rows x one segment in shared memory for coalesced
// access; column kernels give each lane one column.
// ---------------------------------------------------------------------------
constexpr int kSeg = kDirSeg;
constexpr int kTileCols = 2 * kSeg;

__device__ __forceinline__ int seg_count(int n) { return n / kSeg > 1 ? n / kSeg : 1; }

__device__ __forceinline__ void fwd_seg(int n, int b, int& lo, int& hi) {
    lo = b * kSeg;
    hi = b == seg_count(n) - 1 ? n : lo + kSeg;
}

__device__ __forceinline__ void bwd_seg(int n, int b, int& lo, int& hi) {
    hi = n - b * kSeg;
    lo = b == seg_count(n) - 1 ? 0 : hi - kSeg;
}

__device__ __forceinline__ double* carry_at(const DirBlurParams& p, int ch, int k, int line, int seg) {
    return p.carry + ((((size_t)ch * kDirMaxComponents + k) * p.lines_max + line) * p.segs_max + seg) * 3;
}

__device__ __forceinline__ double* start_at(const DirBlurParams& p, int ch, int k, int line) {
    return p.start + (((size_t)ch * kDirMaxComponents + k) * p.lines_max + line) * 9;
}

// Entry state of segment seg >= 1: the first segment's true exit, then the map.
__device__ __forceinline__ void scan_entry(const DirComponentDev& c, const DirBlurParams& p, int ch, int k, int line,
                                           int seg, double s[3]) {
    const double* z0 = carry_at(p, ch, k, line, 0);
    s[0] = z0[0];
    s[1] = z0[1];
    s[2] = z0[2];
    for (int i = 1; i < seg; ++i) {
        const double* z = carry_at(p, ch, k, line, i);
        const double a = c.seg[0] * s[0] + c.seg[1] * s[1] + c.seg[2] * s[2] + z[0];
        const double b = c.seg[3] * s[0] + c.seg[4] * s[1] + c.seg[5] * s[2] + z[1];
        const double d = c.seg[6] * s[0] + c.seg[7] * s[1] + c.seg[8] * s[2] + z[2];
        s[0] = a;
        s[1] = b;
        s[2] = d;
    }
}

// Reflected start state from the first `len` samples (the line reads forward from
// `at(0)`): anchor + sum_i w_h[i] (x_i - anchor).
template <typename At>
__device__ __forceinline__ void reflected_start(const double* w, int len, At at, double s[3]) {
    const double anchor = (double)at(0);
    s[0] = s[1] = s[2] = anchor;
    for (int i = 0; i < len; ++i) {
        const double d = (double)at(i) - anchor;
        for (int h = 0; h < 3; ++h) s[h] += w[h * len + i] * d;
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

__device__ __forceinline__ void load_rows(float (*tile)[kTileCols + 1], const float* src, int W, int row0, int H,
                                          int lo, int len) {
    for (int r = 0; r < 32; ++r) {
        const int y = row0 + r;
        for (int c = threadIdx.x; c < len; c += 32) tile[r][c] = y < H ? src[(size_t)y * W + lo + c] : 0.0f;
    }
    __syncwarp();
}

__device__ __forceinline__ void store_rows(float (*tile)[kTileCols + 1], float* dst, int W, int row0, int H, int lo,
                                           int len) {
    __syncwarp();
    for (int r = 0; r < 32; ++r) {
        const int y = row0 + r;
        if (y >= H) break;
        for (int c = threadIdx.x; c < len; c += 32) dst[(size_t)y * W + lo + c] = tile[r][c];
    }
    __syncwarp();
}

// Rows, left to right: exit states (segment 0 from the reflected start).
__global__ void __launch_bounds__(32) dir_rows_partial_fwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    if (seg >= seg_count(W) - 1) return;
    __shared__ float tile[32][kTileCols + 1];
    int lo, hi;
    fwd_seg(W, seg, lo, hi);
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    const float* raw = p.raw[ch];
    load_rows(tile, raw, W, row0, H, lo, hi - lo);
    if (y >= H) return;
    const float* line = raw + (size_t)y * W;
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        double s[3] = {0.0, 0.0, 0.0};
        if (seg == 0) reflected_start(c.h_init, c.h_len, [&](int i) { return line[i]; }, s);
        for (int x = 0; x < hi - lo; ++x) iir_step(c, (double)tile[threadIdx.x][x], s);
        double* z = carry_at(p, ch, k, y, seg);
        z[0] = s[0];
        z[1] = s[1];
        z[2] = s[2];
    }
}

// Rows, left to right: values; the last segment also writes the end block and keeps
// the right-to-left start state.
__global__ void __launch_bounds__(32) dir_rows_final_fwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    __shared__ float in[32][kTileCols + 1];
    __shared__ float out[32][kTileCols + 1];
    int lo, hi;
    fwd_seg(W, seg, lo, hi);
    const int len = hi - lo;
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    const float* raw = p.raw[ch];
    load_rows(in, raw, W, row0, H, lo, len);
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        if (y < H) {
            const float* line = raw + (size_t)y * W;
            double s[3];
            if (seg == 0)
                reflected_start(c.h_init, c.h_len, [&](int i) { return line[i]; }, s);
            else
                scan_entry(c, p, ch, k, y, seg, s);
            for (int x = 0; x < len; ++x) out[threadIdx.x][x] = (float)iir_step(c, (double)in[threadIdx.x][x], s);
            if (seg == seg_count(W) - 1) {
                const int ts = c.h_tsize;
                double term[3] = {0.0, 0.0, 0.0};
                end_block(c.h_term, ts, s, term);
                for (int r = 0; r < ts; ++r)
                    if (len - ts + r >= 0) out[threadIdx.x][len - ts + r] = (float)term[r];
                double* st = start_at(p, ch, k, y);
                for (int h = 0; h < 3; ++h) st[h] = h < ts ? term[h] : s[h];
            }
        }
        store_rows(out, p.temp[ch][k], W, row0, H, lo, len);
    }
}

// Rows, right to left over [0, W - ts): exit states (first segment from the start state).
__global__ void __launch_bounds__(32) dir_rows_partial_bwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    __shared__ float tile[32][kTileCols + 1];
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
            if (seg == 0) {
                const double* st = start_at(p, ch, k, y);
                s[0] = st[0];
                s[1] = st[1];
                s[2] = st[2];
            }
            for (int x = hi - lo - 1; x >= 0; --x) iir_step(c, (double)tile[threadIdx.x][x], s);
            double* z = carry_at(p, ch, k, y, seg);
            z[0] = s[0];
            z[1] = s[1];
            z[2] = s[2];
        }
        __syncwarp();
    }
}

// Rows, right to left: values in place.
__global__ void __launch_bounds__(32) dir_rows_final_bwd_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    __shared__ float tile[32][kTileCols + 1];
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
            if (seg == 0) {
                const double* st = start_at(p, ch, k, y);
                s[0] = st[0];
                s[1] = st[1];
                s[2] = st[2];
            } else {
                scan_entry(c, p, ch, k, y, seg, s);
            }
            for (int x = hi - lo - 1; x >= 0; --x)
                tile[threadIdx.x][x] = (float)iir_step(c, (double)tile[threadIdx.x][x], s);
        }
        store_rows(tile, p.temp[ch][k], W, row0, H, lo, hi - lo);
    }
}

// Columns, first pass from the visual top (memory row H-1) to memory row 0, in place
// over the row-filtered planes: exit states, and the reflected start state (start
// record slots 3..5). Start record: [0..2] the next pass's start state, [3..5] this
// pass's start state, [6..8] the end block.
__global__ void __launch_bounds__(kLineThreads) dir_cols_partial_a_kernel(const __grid_constant__ DirBlurParams p) {
    const int ch = blockIdx.z, seg = blockIdx.y;
    const int W = p.width, H = p.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H)) return;
    int lo, hi;
    bwd_seg(H, seg, lo, hi);
    for (int k = 0; k < p.count; ++k) {
        const DirComponentDev& c = p.comp[k];
        if (c.op != kDirOpYvv) continue;
        const float* T = p.temp[ch][k];
        double s[3] = {0.0, 0.0, 0.0};
        if (seg == 0) {
            // the start reads up to v_len rows above the bottom; they are read here,
            // before the in-place pass rewrites them, and kept for that pass
            reflected_start(c.v_init, c.v_len, [&](int i) { return T[(size_t)(H - 1 - i) * W + x]; }, s);
            double* st = start_at(p, ch, k, x) + 3;
            st[0] = s[0];
            st[1] = s[1];
            st[2] = s[2];
        }
        if (seg >= seg_count(H) - 1) continue;
        for (int y = hi - 1; y >= lo; --y) iir_step(c, (double)T[(size_t)y * W + x], s);
        double* z = carry_at(p, ch, k, x, seg);
        z[0] = s[0];
        z[1] = s[1];
        z[2] = s[2];
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
        if (seg == 0) {
            const double* st = start_at(p, ch, k, x) + 3;
            s[0] = st[0];
            s[1] = st[1];
            s[2] = st[2];
        } else {
            scan_entry(c, p, ch, k, x, seg, s);
        }
        for (int y = hi - 1; y >= lo; --y) {
            const size_t i = (size_t)y * W + x;
            T[i] = (float)iir_step(c, (double)T[i], s);
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
            const double* st = start_at(p, ch, k, x);
            s[0] = st[0];
            s[1] = st[1];
            s[2] = st[2];
            from = c.v_tsize;
        }
        for (int y = from; y < hi; ++y) iir_step(c, (double)T[(size_t)y * W + x], s);
        double* z = carry_at(p, ch, k, x, seg);
        z[0] = s[0];
        z[1] = s[1];
        z[2] = s[2];
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
        if (seg == 0) {
            for (int h = 0; h < 3; ++h) st[k][h] = start[h];
        } else {
            scan_entry(c, p, ch, k, x, seg, st[k]);
        }
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
                for (int o = -c.radius; o <= c.radius; ++o)
                    sum += (double)T[(size_t)reflect_dir(y + o, H) * W + x] * (double)c.taps[o + c.radius];
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

} // namespace

cudaError_t launch_dir_blur(const DirBlurParams& p, cudaStream_t stream) {
    if (p.width <= 0 || p.height <= 0 || p.count <= 0) return cudaSuccess;
    bool fir = false, iir = false;
    for (int k = 0; k < p.count; ++k) {
        fir |= p.comp[k].op == kDirOpFir;
        iir |= p.comp[k].op == kDirOpYvv;
    }
    const int W = p.width, H = p.height;
    const int sw = W / kSeg > 1 ? W / kSeg : 1, sh = H / kSeg > 1 ? H / kSeg : 1;
    const dim3 rows_grid((H + 31) / 32, sw, 3);
    const dim3 cols_grid((W + kLineThreads - 1) / kLineThreads, sh, 3);
    cudaError_t e = cudaSuccess;
    if (fir) {
        const dim3 block(32, 8);
        fjb::count_launch();
        dir_rows_fir_kernel<<<dim3((W + 31) / 32, (H + 7) / 8, 3), block, 0, stream>>>(p);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (iir) {
        fjb::count_launch();
        dir_rows_partial_fwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        fjb::count_launch();
        dir_rows_final_fwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        fjb::count_launch();
        dir_rows_partial_bwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        fjb::count_launch();
        dir_rows_final_bwd_kernel<<<rows_grid, 32, 0, stream>>>(p);
        fjb::count_launch();
        dir_cols_partial_a_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
        fjb::count_launch();
        dir_cols_final_a_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
        fjb::count_launch();
        dir_cols_partial_b_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    fjb::count_launch();
    dir_cols_final_kernel<<<cols_grid, kLineThreads, 0, stream>>>(p);
    return cudaGetLastError();
}

} // namespace fjb
