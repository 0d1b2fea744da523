// fjb_scanner_lut.cu -- scanner PCHIP LUT built on the device in FP64 (a18).
//
// Restates rust/film-juicer-core/src/scanner/lut.rs:108-296: r^3 nodes of
// log2 XYZ seen through the scanner for normalized C/M/Y density, monotone PCHIP
// slopes along each axis, and per-cell min/max clamps. Every FP64 product and sum
// uses the explicitly rounded intrinsics so that no multiply-add is fused, matching
// the host build's two-rounding arithmetic; only pow/log10 may differ from the host
// libm in their last bit.
//
// Four small launches: nodes (one thread per node, 81-lambda loop), slopes (one
// thread per grid line), cells (one thread per cell/channel), packing into the
// 16-byte vectors the render kernel reads.
#include <cuda_runtime.h>

#include "fjb_internal.h"
#include "fjb_launches.h"

namespace fjb {

namespace {

constexpr int kLutThreads = 128;

__global__ void scanner_nodes_kernel(ScannerLutSpec s, ScannerLutDevice out) {
    const int r = s.resolution;
    const int count = r * r * r;
    const int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= count) return;
    const int yi = node % r;
    const int mi = (node / r) % r;
    const int ci = node / (r * r);
    const double top = (double)(r - 1);
    const double nrm[3] = {(double)ci / top, (double)mi / top, (double)yi / top};
    double dens[3];
    for (int c = 0; c < 3; ++c) {
        const double scaled = nrm[c] / (double)s.inverse_span_cmy[c];
        dens[c] = s.medium == 0 ? __dsub_rn(scaled, (double)s.range_min_cmy[c])
                                : __dadd_rn(scaled, (double)s.range_min_cmy[c]);
    }
    double xyz[3] = {0.0, 0.0, 0.0};
    const double* w[3] = {s.wx, s.wy, s.wz};
    for (int k = 0; k < s.k; ++k) {
        const double base = s.baseline ? s.baseline[k] : 0.0;
        double spectral = __dmul_rn(dens[0], s.eps_c[k]);
        spectral = __dadd_rn(spectral, __dmul_rn(dens[1], s.eps_m[k]));
        spectral = __dadd_rn(spectral, __dmul_rn(dens[2], s.eps_y[k]));
        spectral = __dadd_rn(spectral, base);
        const double t = pow(10.0, -spectral);
        for (int c = 0; c < 3; ++c) {
            const double wk = w[c][k];
            if (isfinite(wk)) {
                const double prod = __dmul_rn(t, wk);
                if (!isnan(prod)) xyz[c] = __dadd_rn(xyz[c], prod);
            }
        }
    }
    const double kLog2Of10 = 3.32192809488736234787;
    for (int c = 0; c < 3; ++c) {
        const double sum = __dmul_rn(xyz[c], s.inv_yn);
        const double lg = log10(__dadd_rn(fmax(sum, 0.0), 1e-10));
        const double v = __dmul_rn(lg, kLog2Of10);
        if (!isfinite(lg)) atomicOr(out.failure, 1u);
        out.nodes[node * 3 + c] = v;
        out.log2_xyz[node * 3 + c] = (float)v;
    }
}

__device__ __forceinline__ double pchip_end(double a, double b) {
    const double slope = __dmul_rn(0.5, __dsub_rn(__dmul_rn(3.0, a), b));
    if (__dmul_rn(slope, a) <= 0.0) return 0.0;
    if (__dmul_rn(a, b) < 0.0 && fabs(slope) > fabs(__dmul_rn(3.0, a))) return __dmul_rn(3.0, a);
    return slope;
}

// One thread per (axis, a, b, channel) line.
__global__ void scanner_slopes_kernel(int r, const double* __restrict__ nodes, float* sc, float* sm, float* sy) {
    const int lines = 3 * r * r * 3;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= lines) return;
    const int channel = id % 3;
    const int b = (id / 3) % r;
    const int a = (id / (3 * r)) % r;
    const int axis = id / (3 * r * r);
    float* out = axis == 0 ? sc : (axis == 1 ? sm : sy);
    auto point = [&](int i) {
        int c, m, y;
        if (axis == 0) {
            c = i; m = a; y = b;
        } else if (axis == 1) {
            c = a; m = i; y = b;
        } else {
            c = a; m = b; y = i;
        }
        return (((c * r + m) * r + y) * 3) + channel;
    };
    if (r == 2) {
        const double d0 = __dsub_rn(nodes[point(1)], nodes[point(0)]);
        out[point(0)] = (float)d0;
        out[point(1)] = (float)d0;
        return;
    }
    double prev = __dsub_rn(nodes[point(1)], nodes[point(0)]);
    const double second = __dsub_rn(nodes[point(2)], nodes[point(1)]);
    out[point(0)] = (float)pchip_end(prev, second);
    double last_minus_one = prev;
    for (int i = 1; i < r - 1; ++i) {
        const double next = __dsub_rn(nodes[point(i + 1)], nodes[point(i)]);
        double slope;
        if (prev == 0.0 || next == 0.0 || __dmul_rn(prev, next) <= 0.0) {
            slope = 0.0;
        } else {
            slope = __ddiv_rn(__dmul_rn(__dmul_rn(2.0, prev), next), __dadd_rn(prev, next));
        }
        out[point(i)] = (float)slope;
        last_minus_one = prev;
        prev = next;
    }
    // prev is delta[r-2], last_minus_one is delta[r-3]
    out[point(r - 1)] = (float)pchip_end(prev, last_minus_one);
}

__global__ void scanner_cells_kernel(int r, const double* __restrict__ nodes, float* cmin, float* cmax) {
    const int s = r - 1;
    const int total = s * s * s * 3;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= total) return;
    const int channel = id % 3;
    const int cell = id / 3;
    const int y = cell % s;
    const int m = (cell / s) % s;
    const int c = cell / (s * s);
    auto at = [&](int ci, int mi, int yi) { return nodes[(((ci * r + mi) * r + yi) * 3) + channel]; };
    double lo = at(c, m, y);
    double hi = lo;
    for (int dc = 0; dc < 2; ++dc)
        for (int dm = 0; dm < 2; ++dm)
            for (int dy = 0; dy < 2; ++dy) {
                const double v = at(c + dc, m + dm, y + dy);
                if (v < lo) lo = v;
                if (hi < v) hi = v;
            }
    cmin[id] = (float)lo;
    cmax[id] = (float)hi;
}

__global__ void scanner_pack_kernel(ScannerLutDevice out, int r) {
    const int nodeCount = r * r * r * 3;
    const int s = r - 1;
    const int cellCount = s * s * s;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < nodeCount) {
        out.packed_nodes[id] = make_float4(out.log2_xyz[id], out.slope_c[id], out.slope_m[id], out.slope_y[id]);
    }
    if (id < cellCount) {
        const float* lo = out.cell_min + 3 * id;
        const float* hi = out.cell_max + 3 * id;
        out.packed_cells[2 * id] = make_float4(lo[0], lo[1], lo[2], hi[0]);
        out.packed_cells[2 * id + 1] = make_float4(hi[1], hi[2], 0.0f, 0.0f);
    }
}

} // namespace

cudaError_t launch_scanner_lut_build(const ScannerLutSpec& spec, const ScannerLutDevice& out, cudaStream_t stream) {
    const int r = spec.resolution;
    if (r < 2 || r > 64 || spec.k <= 0) return cudaErrorInvalidValue;
    const int nodes = r * r * r;
    fjb::count_launch();
    scanner_nodes_kernel<<<(nodes + kLutThreads - 1) / kLutThreads, kLutThreads, 0, stream>>>(spec, out);
    const int lines = 3 * r * r * 3;
    fjb::count_launch();
    scanner_slopes_kernel<<<(lines + kLutThreads - 1) / kLutThreads, kLutThreads, 0, stream>>>(
        r, out.nodes, out.slope_c, out.slope_m, out.slope_y);
    const int cells = (r - 1) * (r - 1) * (r - 1) * 3;
    fjb::count_launch();
    scanner_cells_kernel<<<(cells + kLutThreads - 1) / kLutThreads, kLutThreads, 0, stream>>>(r, out.nodes,
                                                                                             out.cell_min, out.cell_max);
    const int packs = nodes * 3;
    fjb::count_launch();
    scanner_pack_kernel<<<(packs + kLutThreads - 1) / kLutThreads, kLutThreads, 0, stream>>>(out, r);
    return cudaGetLastError();
}

} // namespace fjb
