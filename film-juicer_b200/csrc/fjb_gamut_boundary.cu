// fjb_gamut_boundary.cu -- the output gamut boundary (cmax) table built on the device.
//
// Restates rust/film-juicer-core/src/gamut.rs build_output_boundary (:760-829): for 64
// OkLab lightness rows x 720 hue directions, the three native-RGB channels are cubics in
// chroma (boundary_cubics :727-752); the largest chroma before the first channel leaves
// the slackened unit cube (first_channel_exit :684-726: derivative roots partition the
// chroma range, 20 bisections in the first partition whose end is outside) is the
// table's entry. All FP64 arithmetic is spelled out unfused (__dmul_rn / __dadd_rn /
// __ddiv_rn / __dsqrt_rn), as the Rust host evaluates it, so the table is the
// reference's word for word; the hue directions' cos / sin come from the host's C
// library, as in the Rust build. One thread per table entry.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/juicer_b200.h"
#include "fjb_launches.h"
#include "fjb_schedule.h"

namespace fjb {

namespace {

constexpr int kLightness = 64, kHues = 720;
// Failures are reported as the reference does: the first failing entry in (lightness,
// hue) order, and within an entry the endpoint test before the first-exit test. Each
// failing entry offers the key 2 * index + (0 endpoint inside | 1 exit not finite);
// the smallest key wins.
constexpr unsigned kNoFailure = 0xFFFFFFFFu;

// OkLab Lab -> LMS^(1/3) (the reference's f32 literals, gamut.rs:493-503)
__constant__ float kLabToLmsRoot[9] = {1.0f, 0.3963377774f, 0.2158037573f, 1.0f,          -0.1055613458f,
                                       -0.0638541728f, 1.0f, -0.0894841775f, -1.2914855480f};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }

__device__ __forceinline__ double cubic(const double* c, double x) {
    return add(mul(add(mul(add(mul(c[3], x), c[2]), x), c[1]), x), c[0]);
}

__device__ __forceinline__ bool inside(double v) {
    const double slack = (double)1e-6f;
    return isfinite(v) && v >= -slack && v <= add(1.0, slack);
}

__device__ void derivative_roots(const double* c, double* parts, int& n) {
    const double a = mul(3.0, c[3]), b = mul(2.0, c[2]), cc = c[1];
    auto push = [&](double r) {
        if (isfinite(r) && r > 0.0 && r < 2.0) parts[n++] = r;
    };
    double scale = fabs(a);
    const double vals[3] = {fabs(b), fabs(cc), 1.0};
    for (double v : vals)
        if (scale < v) scale = v;
    const double tol = mul(1e-14, scale);
    if (fabs(a) <= tol) {
        if (fabs(b) > tol) push(__ddiv_rn(-cc, b));
        return;
    }
    const double disc = add(mul(b, b), -mul(mul(4.0, a), cc));
    if (!(disc >= 0.0)) return;
    const double q = mul(-0.5, add(b, copysign(__dsqrt_rn(disc), b)));
    if (fabs(q) <= tol) {
        push(__ddiv_rn(-b, mul(2.0, a)));
        return;
    }
    push(__ddiv_rn(q, a));
    push(__ddiv_rn(cc, q));
}

__device__ double first_exit(const double* c) {
    if (!inside(cubic(c, 0.0))) return 0.0;
    double p[4] = {0.0, 2.0, 0.0, 0.0};
    int n = 2;
    derivative_roots(c, p, n);
    for (int i = 1; i < n; ++i) {
        const double v = p[i];
        int j = i;
        while (j > 0 && v < p[j - 1]) {
            p[j] = p[j - 1];
            --j;
        }
        p[j] = v;
    }
    int kept = 1;
    for (int i = 1; i < n; ++i) {
        if (fabs(add(p[kept - 1], -p[i])) <= 1e-12) continue;
        p[kept++] = p[i];
    }
    for (int k = 1; k < kept; ++k) {
        double lo = p[k - 1], hi = p[k];
        if (inside(cubic(c, hi))) continue;
        for (int it = 0; it < 20; ++it) {
            const double mid = mul(0.5, add(lo, hi));
            if (inside(cubic(c, mid)))
                lo = mid;
            else
                hi = mid;
        }
        return lo;
    }
    return INFINITY;
}

struct BoundaryParams {
    double m[9];
    double dir[kHues][2];
};

__global__ void __launch_bounds__(128) boundary_kernel(const BoundaryParams* __restrict__ p, float* cmax,
                                                       unsigned* flags) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= kLightness * kHues) return;
    const int li = idx / kHues, hi = idx - li * kHues;
    const double lmin = (double)0.02f, lmax = (double)1.0f;
    const double light = add(lmin, __ddiv_rn(mul(add(lmax, -lmin), (double)li), (double)(kLightness - 1)));
    const double dc = p->dir[hi][0], ds = p->dir[hi][1];
    double u[3], v[3];
    for (int r = 0; r < 3; ++r) {
        u[r] = mul((double)kLabToLmsRoot[r * 3], light);
        v[r] = add(mul((double)kLabToLmsRoot[r * 3 + 1], dc), mul((double)kLabToLmsRoot[r * 3 + 2], ds));
    }
    bool end_out = false, neutral_in = true;
    double fe = INFINITY;
    for (int ch = 0; ch < 3; ++ch) {
        double c[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < 3; ++k) {
            const double w = p->m[ch * 3 + k];
            c[0] = add(c[0], mul(mul(mul(w, u[k]), u[k]), u[k]));
            c[1] = add(c[1], mul(mul(mul(mul(w, 3.0), u[k]), u[k]), v[k]));
            c[2] = add(c[2], mul(mul(mul(mul(w, 3.0), u[k]), v[k]), v[k]));
            c[3] = add(c[3], mul(mul(mul(w, v[k]), v[k]), v[k]));
        }
        neutral_in = neutral_in && inside(cubic(c, 0.0));
        end_out = end_out || !inside(cubic(c, 2.0));
        const double e = first_exit(c);
        if (e < fe) fe = e;
    }
    if (!neutral_in) fe = 0.0;
    if (!end_out)
        atomicMin(flags, 2u * (unsigned)idx);
    else if (!(isfinite(fe) && fe >= 0.0 && fe <= 2.0))
        atomicMin(flags, 2u * (unsigned)idx + 1u);
    cmax[idx] = (float)fe;
}

} // namespace

} // namespace fjb

extern "C" FjStatus fjb_gamut_boundary_build(const double* lms_to_native, float* cmax, void* stream,
                                             FjErrorBuffer* error) {
    using namespace fjb;
    try {
        if (!lms_to_native || !cmax) return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "null argument");
        BoundaryParams h{};
        for (int i = 0; i < 9; ++i) h.m[i] = lms_to_native[i];
        const double two_pi = 6.283185307179586476925286766559;
        for (int i = 0; i < kHues; ++i) {
            const double hue = -0.5 * two_pi + two_pi * (double)i / (double)kHues;
            h.dir[i][0] = std::cos(hue);
            h.dir[i][1] = std::sin(hue);
        }
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        // parameters and flags for the call: allocated, freed before it returns
        void* scratch = nullptr;
        cudaError_t e = cudaMalloc(&scratch, sizeof(BoundaryParams) + 256);
        if (e != cudaSuccess) return cuda_status(e, error, "gamut boundary scratch");
        BoundaryParams* dp = static_cast<BoundaryParams*>(scratch);
        unsigned* flags = reinterpret_cast<unsigned*>(static_cast<char*>(scratch) + sizeof(BoundaryParams));
        unsigned f = kNoFailure;
        // pageable source: the copy completes before cudaMemcpyAsync returns
        e = cudaMemcpyAsync(dp, &h, sizeof(h), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0xFF, sizeof(unsigned), s);
        if (e == cudaSuccess) {
            fjb::count_launch();
            boundary_kernel<<<(kLightness * kHues + 127) / 128, 128, 0, s>>>(dp, cmax, flags);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&f, flags, sizeof(f), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(scratch);
        if (e != cudaSuccess) return cuda_status(e, error, "gamut boundary build");
        if (f != kNoFailure) {
            if (f & 1u)
                return fail_status(FJ_STATUS_PREPARATION_FAILURE, error,
                                   "gamut boundary: requirement=finite_first_exit");
            char text[128];
            const unsigned idx = f >> 1;
            std::snprintf(text, sizeof text, "gamut boundary: requirement=c2_outside lightness_index=%u hue_index=%u",
                          idx / kHues, idx % kHues);
            return fail_status(FJ_STATUS_PREPARATION_FAILURE, error, text);
        }
        write_error(error, "");
        return ok_status();
    } catch (...) {
        return fail_status(FJ_STATUS_INTERNAL_FAILURE, error, "unexpected exception in fjb_gamut_boundary_build");
    }
}
