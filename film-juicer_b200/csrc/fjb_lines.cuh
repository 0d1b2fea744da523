// fjb_lines.cuh -- third-order linear recursions over whole lines held in shared memory.
//
// A CTA stages L lines (rows of a plane, or the columns of a narrow strip) in shared
// memory and runs a recursion along each of them block-parallel: each line is cut
// into segments of kLineSeg samples; thread tasks are (line, segment) pairs.
//   partial : each segment runs from a zero state (segment 0 from the line's entry
//             state) and leaves its exit state;
//   scan    : one thread per line turns the exit states into every segment's entry
//             state: entry_1 = exit_0, entry_{j+1} = M entry_j + exit_j, with M the
//             recursion's state map over one segment (FP64);
//   final   : each segment runs again from its entry state, writing in place.
// In exact arithmetic this equals the sequential recursion; in floating point it
// differs from it by rounding. Layout: element i of a line sits at
// (i / kLineSeg) * (kLineSeg + 1) + i % kLineSeg (times the element stride), so that
// the threads of a warp, which walk different segments in step, hit different banks.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fjb {
namespace lines {

constexpr int kLineSeg = 64;
constexpr int kSegStride = kLineSeg + 1;

__host__ __device__ __forceinline__ int segs(int n) { return (n + kLineSeg - 1) / kLineSeg; }
__host__ __device__ __forceinline__ int padded(int n) { return segs(n) * kSegStride; }
__device__ __forceinline__ int at(int i) { return (i / kLineSeg) * kSegStride + i % kLineSeg; }

// Length of segment j of an n-sample line, and the line position of its t-th sample
// (forward: ascending from 64 j; backward: descending from n-1-64 j).
__device__ __forceinline__ int seg_len(int n, int j) {
    const int rest = n - j * kLineSeg;
    return rest < kLineSeg ? rest : kLineSeg;
}
__device__ __forceinline__ int seg_pos(int n, int j, int t, bool forward) {
    return forward ? j * kLineSeg + t : n - 1 - j * kLineSeg - t;
}

// Runs segment j of a line (positions [off, off + n), forward or backward) from state
// s. Samples are read kChunk at a time into registers, so each chunk pays the shared
// memory latency once, then stepped (and written back in place when kWrite).
template <bool kWrite, typename Step>
__device__ __forceinline__ void run_segment(const Step& op, float* b, int es, int n, int j, bool forward, int off,
                                            typename Step::Real s[3]) {
    constexpr int kChunk = 8;
    const int len = seg_len(n, j);
    for (int t0 = 0; t0 < len; t0 += kChunk) {
        float x[kChunk];
        int idx[kChunk];
#pragma unroll
        for (int k = 0; k < kChunk; ++k) {
            const int t = t0 + k < len ? t0 + k : len - 1; // past the end: re-read the last sample
            idx[k] = at(off + seg_pos(n, j, t, forward)) * es;
            x[k] = b[idx[k]];
        }
#pragma unroll
        for (int k = 0; k < kChunk; ++k) {
            if (t0 + k < len) {
                const auto v = op.step(x[k], s);
                if (kWrite) b[idx[k]] = (float)v;
            }
        }
    }
}

// One direction over all L lines of the CTA. `Step` provides
//   using Real;                               // state precision
//   Real step(float x, Real s[3]) const;      // one sample, returns the output
//   const double* map() const;                // 3x3 state map over kLineSeg steps
// `buf(line)` returns the line's base pointer (float, element stride `es`), `entry`
// holds each line's entry state (L x 3), `exits` is scratch of L x segs(n) x 3 Real,
// `last` receives each line's final state (may be null). Outputs are written in place
// when `write`. `line_fastest` orders the tasks line-first (column strips, whose lines
// interleave element by element) instead of segment-first (rows), which keeps the
// threads of a warp on different shared-memory banks in both layouts. The recursion
// covers line positions [off, off + n). Caller synchronises before (the line data and
// entry states must be visible) and this function ends with a barrier.
template <typename Step, typename Buf>
__device__ void run_direction(const Step& op, Buf buf, int es, int L, int n, bool forward,
                              const typename Step::Real* entry, typename Step::Real* exits,
                              typename Step::Real* last, bool write, bool line_fastest, int off = 0) {
    using Real = typename Step::Real;
    const int ns = segs(n);
    const int tasks = L * ns;
    // partial
    for (int task = threadIdx.x; task < tasks; task += blockDim.x) {
        const int line = line_fastest ? task % L : task / ns;
        const int j = line_fastest ? task / L : task - line * ns;
        if (j == ns - 1) continue; // its exit state is never used
        Real s[3];
        if (j == 0) {
            s[0] = entry[line * 3];
            s[1] = entry[line * 3 + 1];
            s[2] = entry[line * 3 + 2];
        } else {
            s[0] = s[1] = s[2] = Real(0);
        }
        run_segment<false>(op, buf(line), es, n, j, forward, off, s);
        Real* e = exits + ((size_t)line * ns + j) * 3;
        e[0] = s[0];
        e[1] = s[1];
        e[2] = s[2];
    }
    __syncthreads();
    // scan
    const double* M = op.map();
    for (int line = threadIdx.x; line < L; line += blockDim.x) {
        if (ns < 2) continue;
        Real* e = exits + (size_t)line * ns * 3;
        double a = e[0], b = e[1], c = e[2];
        for (int j = 1; j < ns; ++j) {
            double za = 0.0, zb = 0.0, zc = 0.0;
            if (j < ns - 1) {
                za = e[j * 3];
                zb = e[j * 3 + 1];
                zc = e[j * 3 + 2];
            }
            e[j * 3] = (Real)a;
            e[j * 3 + 1] = (Real)b;
            e[j * 3 + 2] = (Real)c;
            const double na = M[0] * a + M[1] * b + M[2] * c + za;
            const double nb = M[3] * a + M[4] * b + M[5] * c + zb;
            const double nc = M[6] * a + M[7] * b + M[8] * c + zc;
            a = na;
            b = nb;
            c = nc;
        }
    }
    __syncthreads();
    // final
    for (int task = threadIdx.x; task < tasks; task += blockDim.x) {
        const int line = line_fastest ? task % L : task / ns;
        const int j = line_fastest ? task / L : task - line * ns;
        Real s[3];
        const Real* e = j == 0 ? entry + line * 3 : exits + ((size_t)line * ns + j) * 3;
        s[0] = e[0];
        s[1] = e[1];
        s[2] = e[2];
        if (write)
            run_segment<true>(op, buf(line), es, n, j, forward, off, s);
        else
            run_segment<false>(op, buf(line), es, n, j, forward, off, s);
        if (last && j == ns - 1) {
            last[line * 3] = s[0];
            last[line * 3 + 1] = s[1];
            last[line * 3 + 2] = s[2];
        }
    }
    __syncthreads();
}

// Threads for a CTA that runs L lines of n samples: one per (line, segment) task,
// rounded to whole warps, within [128, kMaxLineThreads].
constexpr int kMaxLineThreads = 512;
inline int line_threads(int L, int n) {
    const int t = (L * segs(n) + 31) / 32 * 32;
    return t < 128 ? 128 : (t > kMaxLineThreads ? kMaxLineThreads : t);
}

// Stages rows [row0, row0 + L) of a row-major plane (`stride` floats per row, W
// columns) into the padded line layout at dst + r * padded(W): 4-byte cp.async copies,
// all in flight at once. Ends with a barrier.
__device__ __forceinline__ void load_rows(float* dst, const float* src, long long stride, int row0, int L, int W) {
    const int pw = padded(W);
    for (int i = threadIdx.x; i < L * W; i += blockDim.x) {
        const int r = i / W, x = i - r * W;
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst + (size_t)r * pw + at(x));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src + (long long)(row0 + r) * stride + x));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
}

// Stages a strip of `C` <= 8 columns starting at column x0 of a row-major plane (W
// floats per row, H rows) into `work` (element (y, c) at at(y) * 8 + c). Full,
// 16-byte aligned strips go through cp.async (two 16-byte copies per row, all in
// flight at once); others through plain loads. Ends with a barrier.
__device__ __forceinline__ void load_strip8(float* work, const float* T, long long W, int H, int x0, int C) {
    const bool aligned = C == 8 && (W % 4) == 0 && (reinterpret_cast<uintptr_t>(T) % 16) == 0;
    if (aligned) {
        for (int i = threadIdx.x; i < H * 2; i += blockDim.x) {
            const int y = i >> 1, h = i & 1;
            const float* src = T + (long long)y * W + x0 + 4 * h;
            const unsigned dst = (unsigned)__cvta_generic_to_shared(work + at(y) * 8 + 4 * h);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
        }
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group 0;\n" ::);
    } else {
        for (int i = threadIdx.x; i < H * 8; i += blockDim.x) {
            const int y = i >> 3, c = i & 7;
            work[at(y) * 8 + c] = c < C ? T[(long long)y * W + x0 + c] : 0.0f;
        }
    }
    __syncthreads();
}

} // namespace lines
} // namespace fjb
