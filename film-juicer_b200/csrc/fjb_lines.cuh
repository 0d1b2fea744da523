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
//   scan    : the exit states become every piece's entry state: entry_1 = exit_0,
//             entry_{j+1} = M entry_j + exit_j, with M the recursion's state map over
//             kLineSeg steps (FP64), which is exact because every piece between the
//             first and the last is full; evaluated in chunks of four pieces (local
//             folds in parallel, a carry over chunks with M^4, then the fill-in);
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

// Entry states are carried in chunks of kScanChunk pieces; a line of ns pieces has
// scan_chunks(ns) chunks (at least one).
constexpr int kScanChunk = 4;
__host__ __device__ __forceinline__ int scan_chunks(int ns) {
    const int c = (ns - 1 + kScanChunk - 1) / kScanChunk;
    return c > 0 ? c : 1;
}

// One direction over all L lines of the CTA. `Step` provides
//   using Real;                               // state precision
//   Real step(float x, Real s[3]) const;      // one sample, returns the output
//   const double* map() const;                // 3x3 state map over kLineSeg steps
//   const double* map4() const;               // the same over kScanChunk * kLineSeg steps
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
                              typename Step::Real* exits, double* carry, typename Step::Real* last,
                              bool line_fastest) {
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
    // scan, in chunks of kScanChunk entries: (A) each chunk with a successor folds its
    // exit states from zero, (B) one thread per line carries the chunk entry states
    // with the kScanChunk-piece map, (C) each chunk writes its entry states
    const double* M = op.map();
    const double* M4 = op.map4();
    const int nch = scan_chunks(ns);
    for (int task = threadIdx.x; task < L * nch; task += blockDim.x) {
        const int line = task % L, c = task / L;
        if (c >= nch - 1) continue;
        const Real* e = exits + (size_t)line * ns * 3;
        double a = 0.0, b = 0.0, d = 0.0;
#pragma unroll
        for (int t = 0; t < kScanChunk; ++t) {
            const int j = 1 + c * kScanChunk + t; // a full chunk: j <= ns - 2
            const double na = (M[0] * a + M[1] * b) + (M[2] * d + (double)e[j * 3]);
            const double nb = (M[3] * a + M[4] * b) + (M[5] * d + (double)e[j * 3 + 1]);
            const double nd = (M[6] * a + M[7] * b) + (M[8] * d + (double)e[j * 3 + 2]);
            a = na;
            b = nb;
            d = nd;
        }
        double* q = carry + ((size_t)line * nch + c) * 3;
        q[0] = a;
        q[1] = b;
        q[2] = d;
    }
    __syncthreads();
    for (int line = threadIdx.x; line < L; line += blockDim.x) {
        const Real* e = exits + (size_t)line * ns * 3;
        double a = e[0], b = e[1], d = e[2]; // entry of piece 1 = exit of piece 0
        for (int c = 0; c < nch; ++c) {
            double* q = carry + ((size_t)line * nch + c) * 3;
            const double la = q[0], lb = q[1], ld = q[2];
            q[0] = a;
            q[1] = b;
            q[2] = d;
            if (c + 1 < nch) {
                const double na = (M4[0] * a + M4[1] * b) + (M4[2] * d + la);
                const double nb = (M4[3] * a + M4[4] * b) + (M4[5] * d + lb);
                const double nd = (M4[6] * a + M4[7] * b) + (M4[8] * d + ld);
                a = na;
                b = nb;
                d = nd;
            }
        }
    }
    __syncthreads();
    for (int task = threadIdx.x; task < L * nch; task += blockDim.x) {
        const int line = task % L, c = task / L;
        Real* e = exits + (size_t)line * ns * 3;
        const double* q = carry + ((size_t)line * nch + c) * 3;
        double a = q[0], b = q[1], d = q[2];
        for (int t = 0; t < kScanChunk; ++t) {
            const int j = 1 + c * kScanChunk + t;
            if (j >= ns) break;
            double za = 0.0, zb = 0.0, zd = 0.0;
            if (j < ns - 1) {
                za = e[j * 3];
                zb = e[j * 3 + 1];
                zd = e[j * 3 + 2];
            }
            e[j * 3] = (Real)a;
            e[j * 3 + 1] = (Real)b;
            e[j * 3 + 2] = (Real)d;
            const double na = (M[0] * a + M[1] * b) + (M[2] * d + za);
            const double nb = (M[3] * a + M[4] * b) + (M[5] * d + zb);
            const double nd = (M[6] * a + M[7] * b) + (M[8] * d + zd);
            a = na;
            b = nb;
            d = nd;
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

// Stages rows [row0, row0 + L) densely (row r at dst + r * W) for stencils along the
// rows: 16-byte cp.async copies when rows and the plane are 16-byte aligned, else
// 4-byte ones. Ends with a barrier.
__device__ __forceinline__ void load_rows_dense(float* dst, const float* src, long long stride, int row0, int L,
                                                int W) {
    const bool vec = W % 4 == 0 && stride % 4 == 0 && (reinterpret_cast<uintptr_t>(src) & 15u) == 0;
    for (int r = 0; r < L; ++r) {
        const float* row = src + (long long)(row0 + r) * stride;
        const unsigned base = (unsigned)__cvta_generic_to_shared(dst + (size_t)r * W);
        if (vec) {
            for (int x = 4 * threadIdx.x; x < W; x += 4 * blockDim.x)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(base + 4u * (unsigned)x), "l"(row + x));
        } else {
            for (int x = threadIdx.x; x < W; x += blockDim.x)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(base + 4u * (unsigned)x), "l"(row + x));
        }
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
