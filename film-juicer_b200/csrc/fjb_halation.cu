// fjb_halation.cu -- emulsion scatter and halation back-reflection (a16).
//
// Restates src/Cuda/Film/JuicerCudaScatterHalation.cu:690-852 per channel:
//   scatter : plane = (1-a) plane + a ((1-w) G_core(plane) + w sum_i amp_i G_tail_i(plane))
//             (amplitudes 0.1633, 0.6496, 0.1870: src/ScatterHalation.h:59-61)
//   bounce  : plane = plane + s sum_b weight_b G_bounce_b(plane)   [/ (1 + s) if renormalized]
// with each G either identity, a reflect-boundary FIR (radius <= 9) or a 3rd-order
// Young-van Vliet recursion with replicate start (legacy B,B1,B2,B3 or factored
// h,g,t) -- the same operators and pass directions as the reference
// (:29-46 reflect rule, :183-198 recursion steps, :201-282 row passes, :283-345
// column passes).
//
// B200 schedule: the reference runs one read-modify-write accumulation pass per
// Gaussian per channel (up to ~14 full-plane passes per channel). Here every
// Gaussian that reads the same source plane is evaluated in the same sweep: the row
// kernels write one row-filtered plane per Gaussian, and the last column kernel runs
// all column filters of a channel together and applies the scatter/bounce
// combination in its epilogue, so the tail accumulator never touches HBM. All three
// channels run in each launch (grid.z = channel); the recursions are block-parallel
// (below).
#include <cuda_runtime.h>

#include "fjb_launches.h"
#include "fjb_lines.cuh"
#include "fjb_optics.h"

namespace fjb {

namespace {

constexpr int kColThreads = 128;

__device__ __forceinline__ int reflect_half(int i, int n) {
    if (i >= 0 && i < n) return i;
    if (i >= -n && i < 0) return -i - 1;
    if (i >= n && i < 2 * n) return 2 * n - 1 - i;
    const int period = 2 * n;
    i %= period;
    if (i < 0) i += period;
    return i >= n ? period - 1 - i : i;
}

struct YvvState {
    float s1, s2, s3;
};

__device__ __forceinline__ void yvv_init(const OpticGauss& g, float first, YvvState& s) {
    s.s1 = first;
    s.s2 = first;
    s.s3 = g.kind == kGaussYvvFactored ? 0.0f : first;
}

__device__ __forceinline__ float yvv_step(const OpticGauss& g, float x, YvvState& s) {
    if (g.kind == kGaussYvvFactored) {
        s.s1 += g.yvv[0] * (x - s.s1);
        s.s3 = g.yvv[2] * s.s3 + g.yvv[1] * (s.s1 - s.s2);
        s.s2 += s.s3;
        return s.s2;
    }
    // the newest state enters last: the loop-carried dependency is one fused multiply-add
    const float v = __fmaf_rn(g.yvv[1], s.s1, __fmaf_rn(g.yvv[2], s.s2, __fmaf_rn(g.yvv[3], s.s3, g.yvv[0] * x)));
    s.s3 = s.s2;
    s.s2 = s.s1;
    s.s1 = v;
    return v;
}

__host__ __device__ __forceinline__ bool is_yvv(int kind) { return kind == kGaussYvv || kind == kGaussYvvFactored; }

// ---------------------------------------------------------------------------
// Recursive Gaussians, block-parallel. A line is cut into segments of kOpticSeg
// samples (the segment processed last in a direction is shorter, or absorbs a
// remainder of fewer than 8 samples). A partial kernel runs every segment -- the
// first from the line's replicate start, the others from a zero state -- and keeps
// its exit state; a scan kernel turns those into each segment's entry state
// (x_{k+1} = M x_k + Z_k with M the recursion's state map over one segment, in
// FP64); the final kernel runs each segment again from its entry state and writes
// it. In exact arithmetic this is the sequential recursion; in FP32 it differs from
// it by rounding. Row kernels stage 32 rows x one segment in
// shared memory so global accesses stay coalesced; column kernels give each lane one
// column, so a warp reads 32 consecutive floats per step.
// ---------------------------------------------------------------------------
constexpr int kSeg = kOpticSeg;
constexpr int kTileCols = kSeg + 8; // longest segment: a remainder below 8 joins the last one
constexpr int kAhead = 8;           // column kernels: rows loaded ahead of the recursion

__host__ __device__ __forceinline__ int seg_count(int n) {
    if (n <= 0) return 0;
    const int ns = n / kSeg + (n % kSeg >= 8 ? 1 : 0);
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

__device__ __forceinline__ float* carry_at(const OpticPass& P, int job, int g, int line, int seg) {
    return P.carry + ((((size_t)job * kOpticMaxGauss + g) * P.lines_max + line) * P.segs_max + seg) * 3;
}

__device__ __forceinline__ size_t edge_at(const OpticPass& P, int job, int g, int line) {
    return ((size_t)job * kOpticMaxGauss + g) * P.lines_max + line;
}

__device__ __forceinline__ void store_exit(float* c, const YvvState& s) {
    c[0] = s.s1;
    c[1] = s.s2;
    c[2] = s.s3;
}

// Entry state of segment `seg` (processing order): the replicate start from `first`
// for segment 0, else the state the scan kernel left in the carry slot.
__device__ __forceinline__ YvvState entry_state(const OpticGauss& g, const OpticPass& P, int job, int gi, int line,
                                                int seg, float first) {
    YvvState s;
    if (seg == 0) {
        yvv_init(g, first, s);
    } else {
        const float* z = carry_at(P, job, gi, line, seg);
        s = YvvState{z[0], z[1], z[2]};
    }
    return s;
}

enum OpticPassKind : int { kRowsFwd = 0, kRowsBwd = 1, kColsUp = 2, kColsDown = 3 };

// Carry scan of one pass: exit states (segment 0's true, the others from a zero
// state) -> every segment's entry state, in place, in FP64: entry_1 = exit_0,
// entry_{j+1} = M entry_j + Z_j. One thread per (line, job, Gaussian).
__global__ void __launch_bounds__(128) optic_scan_kernel(const __grid_constant__ OpticPass P, int pass) {
    const int job = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int line = blockIdx.x * blockDim.x + threadIdx.x;
    const bool rows = pass == kRowsFwd || pass == kRowsBwd;
    if (line >= (rows ? P.height : P.width)) return;
    const int ns = seg_count(rows ? P.width : P.height);
    if (ns < 2) return;
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        const float* z0 = carry_at(P, job, gi, line, 0);
        double a = z0[0], b = z0[1], c = z0[2];
        // exit states are loaded a batch ahead of the dependent chain and the entry
        // stores (the loads cannot pass the stores to the same buffer otherwise)
        constexpr int B = 8;
        float nz[B][3];
        auto load_batch = [&](int j0) {
#pragma unroll
            for (int t = 0; t < B; ++t) {
                const int j = j0 + t;
                if (j < ns - 1) {
                    const float* z = carry_at(P, job, gi, line, j);
                    nz[t][0] = z[0];
                    nz[t][1] = z[1];
                    nz[t][2] = z[2];
                } else {
                    nz[t][0] = nz[t][1] = nz[t][2] = 0.0f; // the last segment keeps no exit state
                }
            }
        };
        load_batch(1);
        for (int j0 = 1; j0 < ns; j0 += B) {
            float z[B][3];
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
                float* slot = carry_at(P, job, gi, line, j);
                slot[0] = (float)a;
                slot[1] = (float)b;
                slot[2] = (float)c;
                const double na = g.seg[0] * a + g.seg[1] * b + g.seg[2] * c + (double)z[t][0];
                const double nb = g.seg[3] * a + g.seg[4] * b + g.seg[5] * c + (double)z[t][1];
                const double nc = g.seg[6] * a + g.seg[7] * b + g.seg[8] * c + (double)z[t][2];
                a = na;
                b = nb;
                c = nc;
            }
        }
    }
}

__device__ __forceinline__ void load_rows(float (*tile)[kTileCols + 1], const float* src, long long stride, int row0,
                                          int H, int lo, int len) {
    for (int r = 0; r < 32; ++r) {
        const int y = row0 + r;
        for (int c = threadIdx.x; c < len; c += 32) tile[r][c] = y < H ? src[(long long)y * stride + lo + c] : 0.0f;
    }
    __syncwarp();
}

__device__ __forceinline__ void store_rows(float (*tile)[kTileCols + 1], float* dst, long long stride, int row0, int H,
                                           int lo, int len) {
    __syncwarp();
    for (int r = 0; r < 32; ++r) {
        const int y = row0 + r;
        if (y >= H) break;
        for (int c = threadIdx.x; c < len; c += 32) dst[(long long)y * stride + lo + c] = tile[r][c];
    }
    __syncwarp();
}

// Rows, forward, zero-state exit states.
__global__ void __launch_bounds__(32) rows_partial_fwd_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    if (seg >= seg_count(W) - 1) return; // the last segment's exit state is never used
    __shared__ float tile[32][kTileCols + 1];
    int lo, hi;
    fwd_seg(W, seg, lo, hi);
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    load_rows(tile, J.src, J.stride, row0, H, lo, hi - lo);
    if (y >= H) return;
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        YvvState st{0.0f, 0.0f, 0.0f};
        if (seg == 0) yvv_init(g, J.src[(long long)y * J.stride], st);
        for (int c = 0; c < hi - lo; ++c) yvv_step(g, tile[threadIdx.x][c], st);
        store_exit(carry_at(P, job, gi, y, seg), st);
    }
}

// Rows, forward, final values into the Gaussian's row-filtered plane.
__global__ void __launch_bounds__(32) rows_final_fwd_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    if (seg >= seg_count(W)) return;
    __shared__ float tile[32][kTileCols + 1];
    int lo, hi;
    fwd_seg(W, seg, lo, hi);
    const int len = hi - lo;
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        load_rows(tile, J.src, J.stride, row0, H, lo, len);
        if (y < H) {
            YvvState st = entry_state(g, P, job, gi, y, seg, J.src[(long long)y * J.stride]);
            for (int c = 0; c < len; ++c) tile[threadIdx.x][c] = yvv_step(g, tile[threadIdx.x][c], st);
            if (seg == seg_count(W) - 1) P.edge_a[edge_at(P, job, gi, y)] = tile[threadIdx.x][len - 1];
        }
        store_rows(tile, J.temp[gi], W, row0, H, lo, len);
    }
}

// Rows, backward, zero-state exit states over the forward result.
__global__ void __launch_bounds__(32) rows_partial_bwd_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    if (seg >= seg_count(W) - 1) return;
    __shared__ float tile[32][kTileCols + 1];
    int lo, hi;
    bwd_seg(W, seg, lo, hi);
    const int len = hi - lo;
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        load_rows(tile, J.temp[gi], W, row0, H, lo, len);
        if (y < H) {
            YvvState st{0.0f, 0.0f, 0.0f};
            if (seg == 0) yvv_init(g, P.edge_a[edge_at(P, job, gi, y)], st);
            for (int c = len - 1; c >= 0; --c) yvv_step(g, tile[threadIdx.x][c], st);
            store_exit(carry_at(P, job, gi, y, seg), st);
        }
        __syncwarp();
    }
}

// Rows, backward, final values in place.
__global__ void __launch_bounds__(32) rows_final_bwd_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    if (seg >= seg_count(W)) return;
    __shared__ float tile[32][kTileCols + 1];
    int lo, hi;
    bwd_seg(W, seg, lo, hi);
    const int len = hi - lo;
    const int row0 = blockIdx.x * 32, y = row0 + threadIdx.x;
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        load_rows(tile, J.temp[gi], W, row0, H, lo, len);
        if (y < H) {
            YvvState st = entry_state(g, P, job, gi, y, seg, P.edge_a[edge_at(P, job, gi, y)]);
            for (int c = len - 1; c >= 0; --c) tile[threadIdx.x][c] = yvv_step(g, tile[threadIdx.x][c], st);
        }
        store_rows(tile, J.temp[gi], W, row0, H, lo, len);
    }
}

// Row pass, FIR Gaussians (reflect boundary): one thread per output pixel.
__global__ void rows_fir_kernel(const __grid_constant__ OpticPass P) {
    const OpticJob& J = P.job[blockIdx.z];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= P.width || y >= P.height) return;
    const float* row = J.src + (long long)y * J.stride;
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (g.kind != kGaussFir) continue;
        float sum = 0.0f;
        if (x - g.radius >= 0 && x + g.radius < P.width)
            for (int o = -g.radius; o <= g.radius; ++o) sum += row[x + o] * g.w[o + g.radius];
        else
            for (int o = -g.radius; o <= g.radius; ++o) sum += row[reflect_half(x + o, P.width)] * g.w[o + g.radius];
        J.temp[gi][(long long)y * P.width + x] = sum;
    }
}

// ---------------------------------------------------------------------------
// Columns: the recursive Gaussians run bottom-up first (the reference's
// anticausal-first column order) in place over the row-filtered planes, then top-down
// fused with the combination: each thread owns one column segment and evaluates every
// Gaussian at each of its pixels, then applies the scatter/bounce combination.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kColThreads) cols_partial_up_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H)) return;
    int lo, hi;
    bwd_seg(H, seg, lo, hi);
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        const float* T = J.temp[gi];
        YvvState st{0.0f, 0.0f, 0.0f};
        if (seg == 0) {
            const float bottom = T[(long long)(H - 1) * W + x];
            P.edge_a[edge_at(P, job, gi, x)] = bottom;
            yvv_init(g, bottom, st);
        }
        if (seg == seg_count(H) - 1) continue;
        for (int y0 = hi - 1; y0 >= lo; y0 -= kAhead) {
            float v[kAhead];
#pragma unroll
            for (int r = 0; r < kAhead; ++r) v[r] = y0 - r >= lo ? T[(long long)(y0 - r) * W + x] : 0.0f;
#pragma unroll
            for (int r = 0; r < kAhead; ++r)
                if (y0 - r >= lo) yvv_step(g, v[r], st);
        }
        store_exit(carry_at(P, job, gi, x, seg), st);
    }
}

__global__ void __launch_bounds__(kColThreads) cols_final_up_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H)) return;
    int lo, hi;
    bwd_seg(H, seg, lo, hi);
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        float* T = J.temp[gi];
        YvvState st = entry_state(g, P, job, gi, x, seg, P.edge_a[edge_at(P, job, gi, x)]);
        for (int y0 = hi - 1; y0 >= lo; y0 -= kAhead) {
            float v[kAhead];
#pragma unroll
            for (int r = 0; r < kAhead; ++r) v[r] = y0 - r >= lo ? T[(long long)(y0 - r) * W + x] : 0.0f;
#pragma unroll
            for (int r = 0; r < kAhead; ++r)
                if (y0 - r >= lo) T[(long long)(y0 - r) * W + x] = yvv_step(g, v[r], st);
        }
        if (lo == 0) P.edge_b[edge_at(P, job, gi, x)] = T[x];
    }
}

__global__ void __launch_bounds__(kColThreads) cols_partial_down_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H) - 1) return;
    int lo, hi;
    fwd_seg(H, seg, lo, hi);
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        const float* T = J.temp[gi];
        YvvState st{0.0f, 0.0f, 0.0f};
        if (seg == 0) yvv_init(g, P.edge_b[edge_at(P, job, gi, x)], st);
        for (int y0 = lo; y0 < hi; y0 += kAhead) {
            float v[kAhead];
#pragma unroll
            for (int r = 0; r < kAhead; ++r) v[r] = y0 + r < hi ? T[(long long)(y0 + r) * W + x] : 0.0f;
#pragma unroll
            for (int r = 0; r < kAhead; ++r)
                if (y0 + r < hi) yvv_step(g, v[r], st);
        }
        store_exit(carry_at(P, job, gi, x, seg), st);
    }
}

__global__ void __launch_bounds__(kColThreads) cols_final_combine_kernel(const __grid_constant__ OpticPass P) {
    const int job = blockIdx.z, seg = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= W || seg >= seg_count(H)) return;
    int lo, hi;
    fwd_seg(H, seg, lo, hi);
    YvvState st[kOpticMaxGauss];
    for (int gi = 0; gi < J.count; ++gi)
        if (is_yvv(J.g[gi].kind)) st[gi] = entry_state(J.g[gi], P, job, gi, x, seg, P.edge_b[edge_at(P, job, gi, x)]);
    for (int y = lo; y < hi; ++y) {
        float v[kOpticMaxGauss];
        for (int gi = 0; gi < J.count; ++gi) {
            const OpticGauss& g = J.g[gi];
            if (g.kind == kGaussIdentity) {
                v[gi] = J.src[(long long)y * J.stride + x];
            } else if (g.kind == kGaussFir) {
                const float* T = J.temp[gi];
                float sum = 0.0f;
                for (int o = -g.radius; o <= g.radius; ++o)
                    sum += T[(long long)reflect_half(y - o, H) * W + x] * g.w[o + g.radius];
                v[gi] = sum;
            } else {
                v[gi] = yvv_step(g, J.temp[gi][(long long)y * W + x], st[gi]);
            }
        }
        float* dst = J.src + (long long)y * J.stride + x;
        const float source = *dst;
        if (J.mode == kOpticScatter) {
            float tail = 0.0f;
            if (J.tail_count > 0) {
                tail = J.coef[0] * v[0];
                for (int i = 1; i < J.tail_count; ++i) tail = tail + J.coef[i] * v[i];
            }
            const float core = v[J.tail_count];
            const float coreTerm = (1.0f - J.tail_weight) * core;
            const float tailTerm = J.tail_weight * tail;
            const float scattered = coreTerm + tailTerm;
            const float sourceTerm = (1.0f - J.amount) * source;
            const float scatteredTerm = J.amount * scattered;
            *dst = sourceTerm + scatteredTerm;
        } else {
            float acc = J.coef[0] * v[0];
            for (int i = 1; i < J.count; ++i) acc = acc + J.coef[i] * v[i];
            const float added = source + J.amount * acc;
            *dst = J.renormalize ? added / (1.0f + J.amount) : added;
        }
    }
}

// ---------------------------------------------------------------------------
// Shared-memory form, used when whole lines fit on chip (the usual case): a CTA
// holds kRowsPerCta full rows, or a kStripCols-wide strip of full columns, and runs
// the block-parallel recursion of fjb_lines.cuh on them, so each Gaussian costs one
// read and one write of the plane per direction pair.
// ---------------------------------------------------------------------------
constexpr int kRowsPerCta = 4;
constexpr int kStripCols = 8;
// CTA sizes (threads, resident CTAs per SM) that bound registers so shared memory,
// not registers, sets the occupancy
constexpr int kRowsThreads = 256, kRowsBlocks = 3;
constexpr int kColsThreads = 288, kColsBlocks = 3;
constexpr size_t kSmemLimit = 200 * 1024;
static_assert(kOpticSeg == lines::kLineSeg, "segment maps are built for the line segment length");

// One recursive Gaussian (kFactored: h, g, t form; else legacy B, B1, B2, B3) with its
// coefficients held in registers (read once per CTA, not once per sample through the
// parameter block).
template <bool kFactored>
struct HalStep {
    using Real = float;
    float c0, c1, c2, c3;
    const double* seg;
    const double* seg4;
    __device__ explicit HalStep(const OpticGauss& g)
        : c0(g.yvv[0]), c1(g.yvv[1]), c2(g.yvv[2]), c3(g.yvv[3]), seg(g.seg), seg4(g.seg4) {}
    __device__ __forceinline__ float step(float x, float s[3]) const {
        if (kFactored) {
            s[0] += c0 * (x - s[0]);
            s[2] = c2 * s[2] + c1 * (s[0] - s[1]);
            s[1] += s[2];
            return s[1];
        }
        const float v = __fmaf_rn(c1, s[0], __fmaf_rn(c2, s[1], __fmaf_rn(c3, s[2], c0 * x)));
        s[2] = s[1];
        s[1] = s[0];
        s[0] = v;
        return v;
    }
    __device__ __forceinline__ const double* map() const { return seg; }
    __device__ __forceinline__ const double* map4() const { return seg4; }
};

// Replicate start of each line from its first sample in processing order (position
// `first`), into entry (L x 3).
template <int ES, typename Buf>
__device__ __forceinline__ void replicate_starts(const OpticGauss& g, Buf buf, int L, int first, float* entry) {
    for (int r = threadIdx.x; r < L; r += blockDim.x) {
        YvvState st;
        yvv_init(g, buf(r)[lines::at(first) * ES], st);
        entry[r * 3] = st.s1;
        entry[r * 3 + 1] = st.s2;
        entry[r * 3 + 2] = st.s3;
    }
    __syncthreads();
}

// Both passes of one recursive Gaussian over L lines of n samples held in shared
// memory: kFirstForward runs ascending positions first (rows: left to right, then
// back), else descending first (columns: bottom-up, then top-down).
template <int ES, bool kFirstForward, bool kFactored, typename Buf>
__device__ __forceinline__ void yvv_lines(const OpticGauss& g, Buf buf, int L, int n, float* exits, double* carry,
                                          float* entry) {
    const HalStep<kFactored> op(g);
    replicate_starts<ES>(g, buf, L, kFirstForward ? 0 : n - 1, entry);
    lines::run_direction<ES, kFirstForward>(op, buf, L, 0, n, entry, exits, carry, (float*)nullptr, ES != 1);
    replicate_starts<ES>(g, buf, L, kFirstForward ? n - 1 : 0, entry);
    lines::run_direction<ES, !kFirstForward>(op, buf, L, 0, n, entry, exits, carry, (float*)nullptr, ES != 1);
}

// Dynamic shared memory: scan carries (doubles) first, then the lines, exit states and
// entry states (floats).
__host__ __device__ inline size_t carry_doubles(int L, int n) { return (size_t)L * lines::scan_chunks(lines::segs(n)) * 3; }

size_t rows_smem_bytes(int W) {
    return carry_doubles(kRowsPerCta, W) * sizeof(double) +
           ((size_t)kRowsPerCta * lines::padded(W) + (size_t)kRowsPerCta * lines::segs(W) * 3 +
            (size_t)kRowsPerCta * 3) *
               sizeof(float);
}

size_t cols_smem_bytes(int H) {
    return carry_doubles(kStripCols, H) * sizeof(double) +
           ((size_t)kStripCols * lines::padded(H) + (size_t)kStripCols * lines::segs(H) * 3 +
            (size_t)kStripCols * 3) *
               sizeof(float);
}

// Rows: every Gaussian of the job into its row-filtered plane (recursive: left to
// right then right to left; FIR: reflect taps).
__global__ void __launch_bounds__(kRowsThreads, kRowsBlocks) rows_smem_kernel(const __grid_constant__ OpticPass P) {
    extern __shared__ __align__(16) float sm[];
    const int job = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    const int row0 = blockIdx.x * kRowsPerCta;
    const int L = min(kRowsPerCta, H - row0);
    const int pw = lines::padded(W);
    double* carry = reinterpret_cast<double*>(sm);
    float* buf = reinterpret_cast<float*>(carry + carry_doubles(kRowsPerCta, W));
    float* exits = buf + (size_t)kRowsPerCta * pw;
    float* entry = exits + (size_t)kRowsPerCta * lines::segs(W) * 3;
    auto line = [&](int r) { return buf + (size_t)r * pw; };
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (g.kind == kGaussFir) {
            // reflect-boundary taps over the densely staged rows
            lines::load_rows_dense(buf, J.src, J.stride, row0, L, W);
            const int rad = g.radius;
            for (int r = 0; r < L; ++r) {
                const float* row = buf + (size_t)r * W;
                float* out = J.temp[gi] + (long long)(row0 + r) * W;
                for (int x = threadIdx.x; x < W; x += blockDim.x) {
                    float sum = 0.0f;
                    if (x - rad >= 0 && x + rad < W)
                        for (int o = -rad; o <= rad; ++o) sum += row[x + o] * g.w[o + rad];
                    else
                        for (int o = -rad; o <= rad; ++o) sum += row[reflect_half(x + o, W)] * g.w[o + rad];
                    out[x] = sum;
                }
            }
            __syncthreads();
            continue;
        }
        if (!is_yvv(g.kind)) continue;
        lines::load_rows(buf, J.src, J.stride, row0, L, W);
        if (g.kind == kGaussYvvFactored)
            yvv_lines<1, true, true>(g, line, L, W, exits, carry, entry);
        else
            yvv_lines<1, true, false>(g, line, L, W, exits, carry, entry);
        lines::store_rows(buf, J.temp[gi], row0, L, W);
    }
}

// Columns of a kStripCols-wide strip: every Gaussian (recursive: bottom-up then
// top-down; FIR: reflect taps; identity) in order, accumulated as the reference
// combines them, then the scatter/bounce combination into the carrier plane. The
// running sum of the Gaussians so far is parked in the strip of the row-filtered plane
// this CTA has just consumed (it stays in L2), which keeps shared memory to one strip.
__global__ void __launch_bounds__(kColsThreads, kColsBlocks) cols_smem_kernel(const __grid_constant__ OpticPass P) {
    extern __shared__ __align__(16) float sm[];
    const int job = blockIdx.y;
    const OpticJob& J = P.job[job];
    const int W = P.width, H = P.height;
    const int x0 = blockIdx.x * kStripCols;
    const int C = min(kStripCols, W - x0);
    const int ph = lines::padded(H);
    double* carry = reinterpret_cast<double*>(sm);
    float* work = reinterpret_cast<float*>(carry + carry_doubles(kStripCols, H)); // [padded(H)][kStripCols]
    float* exits = work + (size_t)ph * kStripCols;
    float* entry = exits + (size_t)kStripCols * lines::segs(H) * 3;
    auto column = [&](int c) { return work + c; };
    const int count = J.count;
    const bool scatter = J.mode == kOpticScatter;
    for (int gi = 0; gi < count; ++gi) {
        const OpticGauss& g = J.g[gi];
        // roles of this Gaussian in the combination
        const bool finishes = scatter ? gi >= J.tail_count : gi == count - 1; // writes the carrier plane
        const bool reads_acc = gi > 0 && (!scatter || J.tail_count > 0);    // a running sum exists
        const bool reads_src = g.kind == kGaussIdentity || finishes;
        const float* acc_in = reads_acc ? J.temp[scatter && finishes ? J.tail_count - 1 : gi - 1] : nullptr;
        float* acc_out = finishes ? nullptr : J.temp[gi];
        // full strips on 16-byte aligned planes move four columns per access
        const bool vec = C == kStripCols && W % 4 == 0 && J.stride % 4 == 0 && lines::aligned16(J.src) &&
                         (g.kind == kGaussIdentity || lines::aligned16(J.temp[gi])) &&
                         (!acc_in || lines::aligned16(acc_in)) && (!acc_out || lines::aligned16(acc_out));
        const bool dense_fir = vec && g.kind == kGaussFir;
        if (dense_fir)
            lines::load_strip8_dense(work, J.temp[gi], W, H, x0);
        else if (g.kind != kGaussIdentity)
            lines::load_strip8(work, J.temp[gi], W, H, x0, C);
        if (g.kind == kGaussYvvFactored)
            yvv_lines<kStripCols, false, true>(g, column, kStripCols, H, exits, carry, entry);
        else if (g.kind == kGaussYvv)
            yvv_lines<kStripCols, false, false>(g, column, kStripCols, H, exits, carry, entry);
        const float coef = J.coef[gi];
        // running sum after this Gaussian, and the carrier value when it finishes the job
        auto running = [&](float v, float a) { return gi == 0 ? coef * v : a + coef * v; };
        auto finish = [&](float v, float a, float source) {
            if (scatter) {
                // the core is the job's last Gaussian
                const float tail = J.tail_count > 0 ? a : 0.0f;
                const float coreTerm = (1.0f - J.tail_weight) * v;
                const float tailTerm = J.tail_weight * tail;
                const float scattered = coreTerm + tailTerm;
                const float sourceTerm = (1.0f - J.amount) * source;
                const float scatteredTerm = J.amount * scattered;
                return sourceTerm + scatteredTerm;
            }
            const float added = source + J.amount * running(v, a);
            return J.renormalize ? added / (1.0f + J.amount) : added;
        };
        if (vec) {
            // thread -> (row, half strip); global reads go kBatch rows at a time
            constexpr int kBatch = 4;
            const int h = threadIdx.x & 1, ys = blockDim.x >> 1;
            for (int y0 = threadIdx.x >> 1; y0 < H; y0 += kBatch * ys) {
                float4 srcv[kBatch], accv[kBatch];
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ys;
                    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    srcv[b] = reads_src && y < H
                                  ? *reinterpret_cast<const float4*>(J.src + (long long)y * J.stride + x0 + 4 * h)
                                  : z;
                    accv[b] = reads_acc && y < H
                                  ? *reinterpret_cast<const float4*>(acc_in + (long long)y * W + x0 + 4 * h)
                                  : z;
                }
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ys;
                    if (y >= H) continue;
                    float4 v;
                    if (g.kind == kGaussIdentity) {
                        v = srcv[b];
                    } else if (g.kind == kGaussFir) {
                        float4 sum = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                        for (int o = -g.radius; o <= g.radius; ++o) {
                            const float4 t = *reinterpret_cast<const float4*>(work + reflect_half(y - o, H) * 8 + 4 * h);
                            const float wt = g.w[o + g.radius];
                            sum.x += t.x * wt;
                            sum.y += t.y * wt;
                            sum.z += t.z * wt;
                            sum.w += t.w * wt;
                        }
                        v = sum;
                    } else {
                        v = *reinterpret_cast<const float4*>(work + lines::at(y) * 8 + 4 * h);
                    }
                    const float4 a = accv[b];
                    if (finishes) {
                        const float4 o4 = make_float4(finish(v.x, a.x, srcv[b].x), finish(v.y, a.y, srcv[b].y),
                                                      finish(v.z, a.z, srcv[b].z), finish(v.w, a.w, srcv[b].w));
                        *reinterpret_cast<float4*>(J.src + (long long)y * J.stride + x0 + 4 * h) = o4;
                    } else {
                        const float4 o4 = make_float4(running(v.x, a.x), running(v.y, a.y), running(v.z, a.z),
                                                      running(v.w, a.w));
                        *reinterpret_cast<float4*>(acc_out + (long long)y * W + x0 + 4 * h) = o4;
                    }
                }
            }
        } else {
            // one column per thread (the block size is a multiple of kStripCols)
            constexpr int kBatch = 8;
            const int c = threadIdx.x % kStripCols, ystep = blockDim.x / kStripCols;
            for (int y0 = threadIdx.x / kStripCols; y0 < H; y0 += kBatch * ystep) {
                float srcv[kBatch], accv[kBatch];
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ystep;
                    const bool in = y < H && c < C;
                    srcv[b] = reads_src && in ? J.src[(long long)y * J.stride + x0 + c] : 0.0f;
                    accv[b] = reads_acc && in ? acc_in[(long long)y * W + x0 + c] : 0.0f;
                }
#pragma unroll
                for (int b = 0; b < kBatch; ++b) {
                    const int y = y0 + b * ystep;
                    if (y >= H || c >= C) continue;
                    float v;
                    if (g.kind == kGaussIdentity) {
                        v = srcv[b];
                    } else if (g.kind == kGaussFir) {
                        float sum = 0.0f;
                        for (int o = -g.radius; o <= g.radius; ++o)
                            sum += work[lines::at(reflect_half(y - o, H)) * kStripCols + c] * g.w[o + g.radius];
                        v = sum;
                    } else {
                        v = work[lines::at(y) * kStripCols + c];
                    }
                    if (finishes)
                        J.src[(long long)y * J.stride + x0 + c] = finish(v, accv[b], srcv[b]);
                    else
                        acc_out[(long long)y * W + x0 + c] = running(v, accv[b]);
                }
            }
        }
        __syncthreads();
    }
}

} // namespace

int optic_segments(int n) { return seg_count(n); }

cudaError_t launch_optic_pass(const OpticPass& P, cudaStream_t stream) {
    if (P.jobs <= 0 || P.width <= 0 || P.height <= 0) return cudaSuccess;
    bool anyYvv = false, anyFir = false;
    for (int j = 0; j < P.jobs; ++j)
        for (int g = 0; g < P.job[j].count; ++g) {
            anyYvv |= is_yvv(P.job[j].g[g].kind);
            anyFir |= P.job[j].g[g].kind == kGaussFir;
        }
    const int W = P.width, H = P.height;
    const int sw = seg_count(W), sh = seg_count(H);
    const dim3 rows_grid((H + 31) / 32, sw, P.jobs);
    const dim3 cols_grid((W + kColThreads - 1) / kColThreads, sh, P.jobs);
    cudaError_t e = cudaSuccess;
    // whole rows / column strips in shared memory when they fit, else the global form
    const size_t rs = rows_smem_bytes(W), cs = cols_smem_bytes(H);
    const bool rows_on_chip = rs <= kSmemLimit, cols_on_chip = cs <= kSmemLimit;
    if ((anyYvv || anyFir) && rows_on_chip) {
        if ((e = cudaFuncSetAttribute(rows_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rs)) !=
            cudaSuccess)
            return e;
        fjb::count_launch();
        rows_smem_kernel<<<dim3((H + kRowsPerCta - 1) / kRowsPerCta, P.jobs), lines::line_threads(kRowsPerCta, W, kRowsThreads), rs,
                           stream>>>(P);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else if (anyYvv) {
        const dim3 row_lines((H + 127) / 128, P.jobs);
        fjb::count_launch();
        rows_partial_fwd_kernel<<<rows_grid, 32, 0, stream>>>(P);
        fjb::count_launch();
        optic_scan_kernel<<<row_lines, 128, 0, stream>>>(P, kRowsFwd);
        fjb::count_launch();
        rows_final_fwd_kernel<<<rows_grid, 32, 0, stream>>>(P);
        fjb::count_launch();
        rows_partial_bwd_kernel<<<rows_grid, 32, 0, stream>>>(P);
        fjb::count_launch();
        optic_scan_kernel<<<row_lines, 128, 0, stream>>>(P, kRowsBwd);
        fjb::count_launch();
        rows_final_bwd_kernel<<<rows_grid, 32, 0, stream>>>(P);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (anyFir && !rows_on_chip) {
        const dim3 block(32, 8);
        fjb::count_launch();
        rows_fir_kernel<<<dim3((W + 31) / 32, (H + 7) / 8, P.jobs), block, 0, stream>>>(P);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (cols_on_chip) {
        if ((e = cudaFuncSetAttribute(cols_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs)) !=
            cudaSuccess)
            return e;
        fjb::count_launch();
        cols_smem_kernel<<<dim3((W + kStripCols - 1) / kStripCols, P.jobs), lines::line_threads(kStripCols, H, kColsThreads), cs,
                           stream>>>(P);
        return cudaGetLastError();
    }
    if (anyYvv) {
        const dim3 col_lines((W + 127) / 128, P.jobs);
        fjb::count_launch();
        cols_partial_up_kernel<<<cols_grid, kColThreads, 0, stream>>>(P);
        fjb::count_launch();
        optic_scan_kernel<<<col_lines, 128, 0, stream>>>(P, kColsUp);
        fjb::count_launch();
        cols_final_up_kernel<<<cols_grid, kColThreads, 0, stream>>>(P);
        fjb::count_launch();
        cols_partial_down_kernel<<<cols_grid, kColThreads, 0, stream>>>(P);
        fjb::count_launch();
        optic_scan_kernel<<<col_lines, 128, 0, stream>>>(P, kColsDown);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    fjb::count_launch();
    cols_final_combine_kernel<<<cols_grid, kColThreads, 0, stream>>>(P);
    return cudaGetLastError();
}

} // namespace fjb
