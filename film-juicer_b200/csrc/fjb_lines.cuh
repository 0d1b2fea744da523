// fjb_lines.cuh -- third-order linear recursions over whole lines held in shared memory.
//
// A CTA stages L lines (rows of a plane, or the columns of a narrow strip) in shared
// memory and runs a recursion along each of them block-parallel. Lines are stored in
// blocks of kLineSeg samples, each followed by one pad word: sample p of a line sits at
// (p / kLineSeg) * (kLineSeg + 1) + p % kLineSeg (times the element stride), so the
// threads of a warp, which walk different blocks in step, hit different banks. A
// recursion over line positions [off, off + n) is cut along those storage blocks
// (only the first and last piece can be shorter than kLineSeg); thread tasks are
// (line, piece) pairs:
//   partial : each piece runs from a zero state (the first from the line's entry
//             state) and leaves its exit state;
//   scan    : one thread per line turns the exit states into every piece's entry
//             state: entry_1 = exit_0, entry_{j+1} = M entry_j + exit_j, with M the
//             recursion's state map over kLineSeg steps (FP64), which is exact
//             because every piece between the first and the last is full;
//   final   : each piece runs again from its entry state, writing in place.
// In exact arithmetic this equals the sequential recursion; in floating point it
// differs from it by rounding.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fjb {
namespace lines {

constexpr int kLineSeg = 64;
constexpr int kSegStride = kLineSeg + 1;

__host__ __device__ __forceinline__ int segs(int n) { return (n + kLineSeg - 1) / kLineSeg; }
__host__ __device__ __forceinline__ int padded(int n) { return segs(n) * kSegStride; }
__device__ __forceinline__ int at(int p) {
    const unsigned u = (unsigned)p;
    return (int)((u / kLineSeg) * kSegStride + u % kLineSeg);
}

// Pieces of the range [off, off + n) (n >= 1), and piece j in processing order:
// storage block q and the block-local sample range [lo, hi).
__device__ __forceinline__ int range_pieces(int off, int n) { return (off + n - 1) / kLineSeg - off / kLineSeg + 1; }
struct Piece {
    int q, lo, hi;
};
template <bool kForward>
__device__ __forceinline__ Piece piece(int off, int n, int j) {
    const int q = kForward ? off / kLineSeg + j : (off + n - 1) / kLineSeg - j;
    const int base = q * kLineSeg;
    const int lo = off > base ? off - base : 0;
    const int end = off + n - base;
    return {q, lo, end < kLineSeg ? end : kLineSeg};
}

// Runs one piece of a line from state s (kForward: ascending positions), writing
// outputs back in place when kWrite. Full pieces read their samples eight at a time
// into registers, so each group pays the shared-memory latency once. ES is the
// element stride of the line in shared memory.
template <bool kWrite, int ES, bool kForward, typename Step>
__device__ __forceinline__ void run_piece(const Step& op, float* line, Piece pc, typename Step::Real s[3]) {
    constexpr int D = kForward ? ES : -ES;
    float* p = line + (pc.q * kSegStride + (kForward ? pc.lo : pc.hi - 1)) * ES;
    const int len = pc.hi - pc.lo;
    if (len == kLineSeg) {
#pragma unroll 1
        for (int c = 0; c < kLineSeg / 8; ++c, p += 8 * D) {
            float x[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = p[k * D];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const auto v = op.step(x[k], s);
                if (kWrite) p[k * D] = (float)v;
            }
        }
    } else {
        // a short first or last piece: one sample at a time
#pragma unroll 1
        for (int t = 0; t < len; ++t, p += D) {
            const auto v = op.step(*p, s);
            if (kWrite) *p = (float)v;
        }
    }
}

// One direction over all L lines of the CTA. `Step` provides
//   using Real;                               // state precision
//   Real step(float x, Real s[3]) const;      // one sample, returns the output
//   const double* map() const;                // 3x3 state map over kLineSeg steps
// `buf(line)` returns the line's base pointer (element stride ES), `entry` holds each
// line's entry state (L x 3), `exits` is scratch of L x segs(off + n) x 3 Real,
// `last` receives each line's final state (may be null). The final pass writes the
// outputs in place. `line_fastest` orders the tasks line-first (column strips, whose lines
// interleave element by element) instead of piece-first (rows), which keeps the
// threads of a warp on different shared-memory banks in both layouts. Caller
// synchronises before (the line data and entry states must be visible) and this
// function ends with a barrier.
template <int ES, bool kForward, typename Step, typename Buf>
__device__ void run_direction(const Step& op, Buf buf, int L, int off, int n, const typename Step::Real* entry,
                              typename Step::Real* exits, typename Step::Real* last, bool line_fastest) {
    using Real = typename Step::Real;
    const int ns = range_pieces(off, n);
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
        run_piece<false, ES, kForward>(op, buf(line), piece<kForward>(off, n, j), s);
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
        run_piece<true, ES, kForward>(op, buf(line), piece<kForward>(off, n, j), s);
        if (last && j == ns - 1) {
            last[line * 3] = s[0];
            last[line * 3 + 1] = s[1];
            last[line * 3 + 2] = s[2];
        }
    }
    __syncthreads();
}

// Threads for a CTA that runs L lines of n samples: one per (line, piece) task,
// rounded to whole warps, within [128, cap] (more tasks loop).
inline int line_threads(int L, int n, int cap) {
    const int t = (L * segs(n) + 31) / 32 * 32;
    return t < 128 ? 128 : (t > cap ? cap : t);
}

// Stages rows [row0, row0 + L) of a row-major plane (`stride` floats per row, W
// columns) into the line layout at dst + r * padded(W): 4-byte cp.async copies, all in
// flight at once. Ends with a barrier.
__device__ __forceinline__ void load_rows(float* dst, const float* src, long long stride, int row0, int L, int W) {
    const int pw = padded(W);
    for (int r = 0; r < L; ++r) {
        const float* row = src + (long long)(row0 + r) * stride;
        const unsigned base = (unsigned)__cvta_generic_to_shared(dst + (size_t)r * pw);
        for (int x = threadIdx.x; x < W; x += blockDim.x)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(base + 4u * (unsigned)at(x)), "l"(row + x));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
}

// Writes rows [row0, row0 + L) back from the line layout (W floats per row of dst).
// Ends with a barrier.
__device__ __forceinline__ void store_rows(const float* buf, float* dst, int row0, int L, int W) {
    const int pw = padded(W);
    for (int r = 0; r < L; ++r) {
        float* row = dst + (long long)(row0 + r) * W;
        const float* line = buf + (size_t)r * pw;
        for (int x = threadIdx.x; x < W; x += blockDim.x) row[x] = line[at(x)];
    }
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

// Stages a full, 16-byte aligned strip of 8 columns densely (element (y, c) at
// y * 8 + c), for stencils that step across rows by a constant offset.
__device__ __forceinline__ void load_strip8_dense(float* work, const float* T, long long W, int H, int x0) {
    for (int i = threadIdx.x; i < H * 2; i += blockDim.x) {
        const int y = i >> 1, h = i & 1;
        const unsigned dst = (unsigned)__cvta_generic_to_shared(work + y * 8 + 4 * h);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(T + (long long)y * W + x0 + 4 * h));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
}

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

} // namespace lines
} // namespace fjb
