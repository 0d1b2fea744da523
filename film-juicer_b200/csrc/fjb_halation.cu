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
// Gaussian that reads the same source plane is evaluated in the same sweep: a row
// kernel writes one row-filtered plane per Gaussian, and a column kernel runs all
// column filters of a channel together and applies the scatter/bounce combination
// in its epilogue, so the tail accumulator never touches HBM. All three channels run
// in one launch (grid.y = channel). Four launches per frame: scatter rows, scatter
// columns + combine, bounce rows, bounce columns + combine.
#include <cuda_runtime.h>

#include "fjb_optics.h"

namespace fjb {

namespace {

constexpr int kTile = 32;     // row kernel: one warp filters 32 rows through 32x32 tiles
constexpr int kColThreads = 128;
constexpr int kPrefetch = 8;  // column kernel: rows loaded ahead of the recursion

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
    const float v = g.yvv[0] * x + g.yvv[1] * s.s1 + g.yvv[2] * s.s2 + g.yvv[3] * s.s3;
    s.s3 = s.s2;
    s.s2 = s.s1;
    s.s1 = v;
    return v;
}

__host__ __device__ __forceinline__ bool is_yvv(int kind) { return kind == kGaussYvv || kind == kGaussYvvFactored; }

// ---------------------------------------------------------------------------
// Row pass, recursive Gaussians: one warp owns 32 rows; 32x32 tiles are staged in
// shared memory so every global access is a coalesced 128-byte row segment, then each
// lane walks its own row through the tile (forward, then backward).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTile) rows_yvv_kernel(const __grid_constant__ OpticPass P) {
    const OpticJob& J = P.job[blockIdx.y];
    __shared__ float tile[kTile][kTile + 1];
    const int lane = threadIdx.x;
    const int row0 = blockIdx.x * kTile;
    if (row0 >= P.height) return;
    const int y = row0 + lane;
    const int W = P.width, H = P.height;
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        float* T = J.temp[gi];
        YvvState st;
        yvv_init(g, y < H ? J.src[(long long)y * J.stride] : 0.0f, st);
        for (int c0 = 0; c0 < W; c0 += kTile) {
            const int x = c0 + lane;
            for (int r = 0; r < kTile; ++r) {
                const int yy = row0 + r;
                tile[r][lane] = (yy < H && x < W) ? J.src[(long long)yy * J.stride + x] : 0.0f;
            }
            __syncwarp();
            const int cols = min(kTile, W - c0);
            for (int c = 0; c < cols; ++c) tile[lane][c] = yvv_step(g, tile[lane][c], st);
            __syncwarp();
            for (int r = 0; r < kTile; ++r) {
                const int yy = row0 + r;
                if (yy < H && x < W) T[(long long)yy * W + x] = tile[r][lane];
            }
            __syncwarp();
        }
        yvv_init(g, y < H ? T[(long long)y * W + W - 1] : 0.0f, st);
        for (int c0 = ((W - 1) / kTile) * kTile; c0 >= 0; c0 -= kTile) {
            const int x = c0 + lane;
            for (int r = 0; r < kTile; ++r) {
                const int yy = row0 + r;
                tile[r][lane] = (yy < H && x < W) ? T[(long long)yy * W + x] : 0.0f;
            }
            __syncwarp();
            const int cols = min(kTile, W - c0);
            for (int c = cols - 1; c >= 0; --c) tile[lane][c] = yvv_step(g, tile[lane][c], st);
            __syncwarp();
            for (int r = 0; r < kTile; ++r) {
                const int yy = row0 + r;
                if (yy < H && x < W) T[(long long)yy * W + x] = tile[r][lane];
            }
            __syncwarp();
        }
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
        for (int o = -g.radius; o <= g.radius; ++o) sum += row[reflect_half(x + o, P.width)] * g.w[o + g.radius];
        J.temp[gi][(long long)y * P.width + x] = sum;
    }
}

// ---------------------------------------------------------------------------
// Column pass + combination. One thread per column: the recursive Gaussians first
// run bottom-up in place (the reference's anticausal-first column order), then a
// single top-down sweep produces every Gaussian's final value at (x, y) and the
// epilogue combines them with the source plane.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float column_value(const OpticJob& J, int gi, const OpticPass& P, int x, int y,
                                              YvvState& st, float tval) {
    const OpticGauss& g = J.g[gi];
    if (g.kind == kGaussIdentity) return J.src[(long long)y * J.stride + x];
    if (g.kind == kGaussFir) {
        const float* T = J.temp[gi];
        float sum = 0.0f;
        for (int o = -g.radius; o <= g.radius; ++o)
            sum += T[(long long)reflect_half(y - o, P.height) * P.width + x] * g.w[o + g.radius];
        return sum;
    }
    return yvv_step(g, tval, st);
}

__global__ void __launch_bounds__(kColThreads) columns_combine_kernel(const __grid_constant__ OpticPass P) {
    const OpticJob& J = P.job[blockIdx.y];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int W = P.width, H = P.height;
    if (x >= W) return;
    // bottom-up pass of every recursive Gaussian, in place
    for (int gi = 0; gi < J.count; ++gi) {
        const OpticGauss& g = J.g[gi];
        if (!is_yvv(g.kind)) continue;
        float* T = J.temp[gi];
        YvvState st;
        yvv_init(g, T[(long long)(H - 1) * W + x], st);
        for (int r0 = H - 1; r0 >= 0; r0 -= kPrefetch) {
            float v[kPrefetch];
#pragma unroll
            for (int r = 0; r < kPrefetch; ++r) v[r] = (r0 - r >= 0) ? T[(long long)(r0 - r) * W + x] : 0.0f;
#pragma unroll
            for (int r = 0; r < kPrefetch; ++r)
                if (r0 - r >= 0) T[(long long)(r0 - r) * W + x] = yvv_step(g, v[r], st);
        }
    }
    YvvState st[kOpticMaxGauss];
    for (int gi = 0; gi < J.count; ++gi)
        if (is_yvv(J.g[gi].kind)) yvv_init(J.g[gi], J.temp[gi][x], st[gi]);
    for (int y = 0; y < H; ++y) {
        float v[kOpticMaxGauss];
        for (int gi = 0; gi < J.count; ++gi) {
            const float t = is_yvv(J.g[gi].kind) ? J.temp[gi][(long long)y * W + x] : 0.0f;
            v[gi] = column_value(J, gi, P, x, y, st[gi], t);
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

} // namespace

cudaError_t launch_optic_pass(const OpticPass& P, cudaStream_t stream) {
    if (P.jobs <= 0 || P.width <= 0 || P.height <= 0) return cudaSuccess;
    bool anyYvv = false, anyFir = false;
    for (int j = 0; j < P.jobs; ++j)
        for (int g = 0; g < P.job[j].count; ++g) {
            anyYvv |= is_yvv(P.job[j].g[g].kind);
            anyFir |= P.job[j].g[g].kind == kGaussFir;
        }
    if (anyYvv) {
        rows_yvv_kernel<<<dim3((P.height + kTile - 1) / kTile, P.jobs), kTile, 0, stream>>>(P);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (anyFir) {
        const dim3 block(32, 8);
        rows_fir_kernel<<<dim3((P.width + 31) / 32, (P.height + 7) / 8, P.jobs), block, 0, stream>>>(P);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    columns_combine_kernel<<<dim3((P.width + kColThreads - 1) / kColThreads, P.jobs), kColThreads, 0, stream>>>(P);
    return cudaGetLastError();
}

} // namespace fjb
