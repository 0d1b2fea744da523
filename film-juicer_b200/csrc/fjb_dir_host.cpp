// fjb_dir_host.cpp -- host preparation of the spatial-DIR operators.
//
// Boundary weights: the reference obtains them from the Rust host
// (native/juicer_dir_boundary_api.h:58-61 -> rust/film-juicer-core/src/film/dir/
// boundary.rs). This file restates that construction with the same double-double
// arithmetic (hi + lo pairs, fused-residual products), so the binary64 outputs match
// the reference's words:
//   start: the causal recursion run over the period-2L reflected extension of the
//          line, i.e. state = (I - A^{2L})^{-1} sum_k (A^k + A^{2L-1-k}) b x_k,
//          truncated once the remaining |weights| fall below the record's accuracy;
//   end:   the anticausal recursion on the last min(L, 3) samples with reflected
//          neighbours, solved as a size x size linear system.
// FIR taps restate rust/film-juicer-core/src/optics/gaussian.rs:16-52.
// Validation restates src/Cuda/Film/JuicerCudaFilmPipeline.cu:860-930 (component
// weights, operator eligibility by sigma, unit DC gain).
#include <cmath>
#include <cstring>

#include "fjb_dir.h"

namespace fjb {

namespace {

// Double-double value hi + lo with the reference's operation sequence (Dekker-style
// sums, fused-residual products; boundary.rs:207-262).
struct Dd {
    double hi = 0.0, lo = 0.0;
    static Dd from(double v) { return Dd{v, 0.0}; }
    static Dd normalize(double hi, double lo) {
        const double sum = hi + lo;
        return Dd{sum, lo - (sum - hi)};
    }
    Dd add(const Dd& r) const {
        const double sum = hi + r.hi;
        const double virt = sum - hi;
        const double err = (hi - (sum - virt)) + (r.hi - virt) + lo + r.lo;
        return normalize(sum, err);
    }
    Dd neg() const { return Dd{-hi, -lo}; }
    Dd sub(const Dd& r) const { return add(r.neg()); }
    Dd mul(const Dd& r) const {
        const double product = hi * r.hi;
        const double err = std::fma(hi, r.hi, -product) + hi * r.lo + lo * r.hi + lo * r.lo;
        return normalize(product, err);
    }
    Dd div(const Dd& d) const {
        const double first = hi / d.hi;
        const Dd rem = sub(d.mul(from(first)));
        const double second = (rem.hi + rem.lo) / d.hi;
        return from(first).add(from(second));
    }
    double value() const { return hi + lo; }
};

using DdMat = Dd[3][3];

void dd_identity(DdMat m) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m[i][j] = Dd::from(i == j ? 1.0 : 0.0);
}

void dd_mul(const DdMat a, const DdMat b, DdMat o) {
    Dd t[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            Dd v = Dd::from(0.0);
            for (int k = 0; k < 3; ++k) v = v.add(a[r][k].mul(b[k][c]));
            t[r][c] = v;
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o[r][c] = t[r][c];
}

void dd_transform(const DdMat m, const Dd v[3], Dd o[3]) {
    Dd t[3];
    for (int r = 0; r < 3; ++r) {
        Dd acc = Dd::from(0.0);
        for (int c = 0; c < 3; ++c) acc = acc.add(m[r][c].mul(v[c]));
        t[r] = acc;
    }
    for (int r = 0; r < 3; ++r) o[r] = t[r];
}

// Gauss-Jordan with partial pivoting on the leading size x size block.
bool dd_invert(DdMat m, int size, DdMat inv) {
    dd_identity(inv);
    for (int col = 0; col < size; ++col) {
        int piv = col;
        double mag = std::fabs(m[piv][col].value());
        for (int r = col + 1; r < size; ++r) {
            const double v = std::fabs(m[r][col].value());
            if (v > mag) {
                piv = r;
                mag = v;
            }
        }
        if (!(mag > 0.0 && std::isfinite(mag))) return false;
        if (piv != col)
            for (int j = 0; j < 3; ++j) {
                std::swap(m[piv][j], m[col][j]);
                std::swap(inv[piv][j], inv[col][j]);
            }
        const Dd scale = m[col][col];
        for (int e = 0; e < size; ++e) {
            m[col][e] = m[col][e].div(scale);
            inv[col][e] = inv[col][e].div(scale);
        }
        for (int r = 0; r < size; ++r) {
            if (r == col) continue;
            const Dd f = m[r][col];
            for (int e = 0; e < size; ++e) {
                m[r][e] = m[r][e].sub(f.mul(m[col][e]));
                inv[r][e] = inv[r][e].sub(f.mul(inv[col][e]));
            }
        }
    }
    return true;
}

long long reflect_period(long long i, long long n) {
    const long long period = 2 * n;
    long long w = i % period;
    if (w < 0) w += period;
    return w < n ? w : period - 1 - w;
}

} // namespace

bool dir_axis_boundary(const FjDirGaussian& g, int L, DirAxisBoundary& out, std::string& why) {
    if (L <= 0 || !(g.boundary_truncation_accuracy > 0.0 && g.boundary_certification_tolerance > 0.0) ||
        g.boundary_derivation_version != 1) {
        why = "spatial DIR boundary policy is invalid";
        return false;
    }
    const double coeff[9] = {g.feedforward, g.feedback[0], g.feedback[1], g.feedback[2], g.normalization_denominator,
                             g.feedforward_numerator, g.feedback_numerators[0], g.feedback_numerators[1],
                             g.feedback_numerators[2]};
    DdMat A;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = Dd::from(0.0);
    for (int c = 0; c < 3; ++c) A[0][c] = Dd::from(coeff[c + 1]);
    A[1][0] = Dd::from(1.0);
    A[2][1] = Dd::from(1.0);
    const long long period = 2LL * L;
    std::vector<Dd> powers((size_t)period * 3);
    powers[0] = Dd::from(coeff[0]);
    for (long long e = 1; e < period; ++e) dd_transform(A, &powers[(size_t)(e - 1) * 3], &powers[(size_t)e * 3]);
    DdMat P;
    dd_identity(P);
    for (long long e = 0; e < period; ++e) dd_mul(A, P, P);
    DdMat S;
    dd_identity(S);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S[i][j] = S[i][j].sub(P[i][j]);
    DdMat Si;
    if (!dd_invert(S, 3, Si)) {
        why = "spatial DIR causal boundary system is singular";
        return false;
    }
    std::vector<double> full((size_t)3 * L);
    Dd sums[3] = {Dd::from(0.0), Dd::from(0.0), Dd::from(0.0)};
    for (int s = 0; s < L; ++s) {
        Dd rhs[3];
        for (int r = 0; r < 3; ++r) rhs[r] = powers[(size_t)s * 3 + r].add(powers[(size_t)(period - 1 - s) * 3 + r]);
        Dd st[3];
        dd_transform(Si, rhs, st);
        for (int r = 0; r < 3; ++r) {
            const double v = st[r].value();
            if (!std::isfinite(v)) {
                why = "spatial DIR boundary weights are not finite";
                return false;
            }
            full[(size_t)r * L + s] = v;
            sums[r] = sums[r].add(Dd::from(v));
        }
    }
    for (int r = 0; r < 3; ++r) {
        const double sum = sums[r].value();
        if (!std::isfinite(sum) || std::fabs(sum - 1.0) > g.boundary_certification_tolerance) {
            why = "spatial DIR boundary weights fail certification";
            return false;
        }
    }
    const int minimum = L < 3 ? L : 3;
    int retained = L;
    double tails[3] = {0, 0, 0};
    for (int s = L - 1; s >= minimum; --s) {
        for (int r = 0; r < 3; ++r) tails[r] += std::fabs(full[(size_t)r * L + s]);
        const double mx = std::fmax(tails[0], std::fmax(tails[1], tails[2]));
        if (mx >= g.boundary_truncation_accuracy) {
            retained = s + 1;
            break;
        }
        retained = s;
    }
    out.length = retained;
    out.weights.assign((size_t)3 * retained, 0.0);
    for (int r = 0; r < 3; ++r)
        for (int s = 0; s < retained; ++s) out.weights[(size_t)r * retained + s] = full[(size_t)r * L + s];
    const int size = L < 3 ? L : 3;
    DdMat T;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[i][j] = Dd::from(0.0);
    for (int d = 0; d < size; ++d) T[d][d] = Dd::from(coeff[4]);
    for (int row = 0; row < size; ++row) {
        const long long oi = (long long)(L - size + row);
        for (int c = 0; c < 3; ++c) {
            const long long refl = reflect_period(oi + c + 1, L);
            const long long col = refl - (L - size);
            if (col < 0 || col >= size) {
                why = "spatial DIR terminal reflection escapes the end block";
                return false;
            }
            T[row][col] = T[row][col].sub(Dd::from(coeff[6 + c]));
        }
    }
    DdMat Ti;
    if (!dd_invert(T, size, Ti)) {
        why = "spatial DIR terminal system is singular";
        return false;
    }
    std::memset(out.terminal, 0, sizeof(out.terminal));
    for (int row = 0; row < size; ++row) {
        double sum = 0.0;
        for (int c = 0; c < size; ++c) {
            const double v = Dd::from(coeff[5]).mul(Ti[row][c]).value();
            out.terminal[row * size + c] = v;
            sum += v;
        }
        if (!std::isfinite(sum) || std::fabs(sum - 1.0) > g.boundary_certification_tolerance) {
            why = "spatial DIR terminal matrix fails certification";
            return false;
        }
    }
    out.terminal_size = size;
    return true;
}

std::vector<float> gaussian_taps(int radius, float sigma_px) {
    std::vector<float> w;
    if (radius < 1 || !(sigma_px > 0.0f) || !std::isfinite(sigma_px)) return w;
    const double sigma = (double)sigma_px;
    const double s2 = sigma * sigma * 2.0;
    double sum = 0.0;
    for (int i = -radius; i <= radius; ++i) {
        const double x = (double)i;
        const double v = std::exp(-(x * x) / s2);
        w.push_back((float)v);
        sum += v;
    }
    const double rec = sum != 0.0 ? 1.0 / sum : 0.0;
    for (float& v : w) v = (float)((double)v * rec);
    return w;
}

void DirPlan::release() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
    count = 0;
}

size_t dir_recursion_bytes(int width, int height) {
    const size_t lines = (size_t)(width > height ? width : height);
    const int sw = dir_segments(width), sh = dir_segments(height);
    const size_t segs = (size_t)(sw > sh ? sw : sh);
    return ((size_t)3 * kDirMaxComponents * lines * segs * 3 + (size_t)3 * kDirMaxComponents * lines * 9) *
           sizeof(double);
}

size_t dir_scratch_floats(int width, int height) {
    // raw corrections (3) + log raw (3) + filtered (3) + one temp per channel/component
    return (size_t)(9 + 3 * kDirMaxComponents) * (size_t)width * (size_t)height;
}

namespace {

void mat3_mul(const double* a, const double* b, double* o) {
    double t[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
    std::memcpy(o, t, sizeof(t));
}

// The recursion 1 / (1 - fb0 z^-1 - fb1 z^-2 - fb2 z^-3) as (1 - p z^-1)(1 - a1 z^-1 -
// a2 z^-2): the real pole p by Newton's method from z = 1 (the Gaussian recursions
// have one real pole in (0, 1) and a complex pair), then the FP32 coefficients
// c0 = 1 - p, c2 = -a2, c1 = 1 - a1 - a2 and, from those rounded values, the basis
// maps and zero-input state maps. In this form the state holds the first-order output,
// the output and its last difference, so FP32 rounding is not amplified by the
// recursion's DC gain as it is in the direct form (about 1 / ff). factored stays 0
// (the FP64 direct form runs) when the coefficients do not have that structure.
void factor_recursion(DirComponentDev& c) {
    c.factored = 0;
    double p = 1.0;
    for (int it = 0; it < 200; ++it) {
        const double f = ((p - c.fb[0]) * p - c.fb[1]) * p - c.fb[2];
        const double d = (3.0 * p - 2.0 * c.fb[0]) * p - c.fb[1];
        if (!(std::fabs(d) > 0.0)) return;
        const double q = p - f / d;
        const bool done = std::fabs(q - p) <= 1e-15 * std::fabs(q);
        p = q;
        if (done) break;
    }
    const double resid = ((p - c.fb[0]) * p - c.fb[1]) * p - c.fb[2];
    if (!(p > 0.0 && p < 1.0) || !(std::fabs(resid) < 1e-12)) return;
    const double a1 = c.fb[0] - p, a2 = c.fb[1] + p * a1;
    const float c0 = (float)(1.0 - p), c2 = (float)(-a2), c1 = (float)(1.0 - a1 - a2);
    if (!(c0 > 0.0f && c1 > 0.0f && c2 > 0.0f && c2 < 1.0f) || !std::isfinite(c1)) return;
    // the rounded coefficients define the FP32 recursion; the maps describe it
    const double P = 1.0 - (double)c0, C1 = c1, C2 = c2, A1 = 1.0 + C2 - C1, A2 = -C2;
    const double T[9] = {1.0 / C1, -A1 / C1, -A2 / C1, 1, 0, 0, 1, -1, 0};
    const double Ti[9] = {0, 1, 0, 0, 1, -1, -C1 / A2, (1.0 - A1) / A2, A1 / A2};
    const double F[9] = {P, 0, 0, C1 * P, 1.0 - C1, C2, C1 * P, -C1, C2};
    double r[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int step = 1; step <= 4 * kDirSeg; ++step) {
        mat3_mul(F, r, r);
        if (step == kDirSeg) std::memcpy(c.seg_f, r, sizeof(r));
    }
    std::memcpy(c.seg4_f, r, sizeof(r));
    std::memcpy(c.to_fac, T, sizeof(T));
    std::memcpy(c.from_fac, Ti, sizeof(Ti));
    c.fac[0] = c0;
    c.fac[1] = c1;
    c.fac[2] = c2;
    c.factored = 1;
}

} // namespace

bool dir_plan_create(const FjSpatialDir& sd, int width, int height, cudaStream_t stream, DirPlan& plan,
                     std::string& why, cudaError_t& err) {
    err = cudaSuccess;
    plan.release();
    plan.width = width;
    plan.height = height;
    if (sd.component_count > (size_t)kDirMaxComponents) {
        why = "spatial DIR has more than four components";
        return false;
    }
    bool any = false;
    int n = 0;
    for (size_t i = 0; i < sd.component_count; ++i) {
        const FjDirGaussian& g = sd.components[i];
        if (!std::isfinite(g.weight) || g.weight < 0.0f) {
            why = "spatial DIR component weight is invalid";
            return false;
        }
        if (!(g.weight > 0.0f)) continue;
        any = true;
        if (!std::isfinite(g.sigma_px) || g.sigma_px < 0.0f) {
            why = "spatial DIR component sigma is invalid";
            return false;
        }
        DirComponentDev c{};
        c.weight = g.weight;
        switch (g.reference_operator) {
            case FJ_DIR_OPERATOR_IDENTITY:
                if (g.radius != 0) {
                    why = "spatial DIR identity component has a radius";
                    return false;
                }
                c.op = kDirOpIdentity;
                break;
            case FJ_DIR_OPERATOR_FIR_REFLECT: {
                if (!(g.sigma_px > 0.0f && g.sigma_px < 3.0f) || g.radius <= 0 || g.radius > kDirMaxFirRadius) {
                    why = "spatial DIR FIR component is malformed";
                    return false;
                }
                c.op = kDirOpFir;
                c.radius = g.radius;
                const std::vector<float> taps = gaussian_taps(g.radius, g.sigma_px);
                void* d = nullptr;
                if ((err = cudaMalloc(&d, taps.size() * sizeof(float))) != cudaSuccess) return false;
                plan.owned.push_back(d);
                if ((err = cudaMemcpyAsync(d, taps.data(), taps.size() * sizeof(float), cudaMemcpyHostToDevice,
                                           stream)) != cudaSuccess)
                    return false;
                if ((err = cudaStreamSynchronize(stream)) != cudaSuccess) return false;
                c.taps = static_cast<const float*>(d);
                c.symmetric_taps = 1;
                for (int i = 0; i <= 2 * g.radius; ++i)
                    if (std::memcmp(&taps[i], &taps[2 * g.radius - i], sizeof(float)) != 0) c.symmetric_taps = 0;
                break;
            }
            case FJ_DIR_OPERATOR_YVV_REFLECT: {
                const double dc = g.feedforward + g.feedback[0] + g.feedback[1] + g.feedback[2];
                if (!(g.sigma_px >= 3.0f) || !std::isfinite(g.feedforward) || !(g.feedforward > 0.0) ||
                    !std::isfinite(g.feedback[0]) || !std::isfinite(g.feedback[1]) || !std::isfinite(g.feedback[2]) ||
                    !std::isfinite(dc) || std::fabs(dc - 1.0) > 1.0e-12) {
                    why = "spatial DIR recursive component is malformed";
                    return false;
                }
                c.op = kDirOpYvv;
                c.ff = g.feedforward;
                for (int k = 0; k < 3; ++k) c.fb[k] = g.feedback[k];
                {
                    // companion map (s0, s1, s2) -> (fb0 s0 + fb1 s1 + fb2 s2, s0, s1) over kDirSeg and 4 kDirSeg steps
                    const double m[9] = {c.fb[0], c.fb[1], c.fb[2], 1, 0, 0, 0, 1, 0};
                    double r[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
                    for (int step = 1; step <= 4 * kDirSeg; ++step) {
                        double t[9];
                        for (int i = 0; i < 3; ++i)
                            for (int j = 0; j < 3; ++j)
                                t[i * 3 + j] = m[i * 3] * r[j] + m[i * 3 + 1] * r[3 + j] + m[i * 3 + 2] * r[6 + j];
                        std::memcpy(r, t, sizeof(r));
                        if (step == kDirSeg) std::memcpy(c.seg, r, sizeof(r));
                    }
                    std::memcpy(c.seg4, r, sizeof(r));
                }
                factor_recursion(c);
                DirAxisBoundary hb, vb;
                if (!dir_axis_boundary(g, width, hb, why) || !dir_axis_boundary(g, height, vb, why)) return false;
                void* d = nullptr;
                const size_t hbytes = hb.weights.size() * sizeof(double), vbytes = vb.weights.size() * sizeof(double);
                if ((err = cudaMalloc(&d, hbytes + vbytes)) != cudaSuccess) return false;
                plan.owned.push_back(d);
                if ((err = cudaMemcpy(d, hb.weights.data(), hbytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
                    (err = cudaMemcpy(static_cast<char*>(d) + hbytes, vb.weights.data(), vbytes,
                                      cudaMemcpyHostToDevice)) != cudaSuccess)
                    return false;
                c.h_init = static_cast<const double*>(d);
                c.h_len = hb.length;
                c.h_tsize = hb.terminal_size;
                std::memcpy(c.h_term, hb.terminal, sizeof(c.h_term));
                c.v_init = reinterpret_cast<const double*>(static_cast<char*>(d) + hbytes);
                c.v_len = vb.length;
                c.v_tsize = vb.terminal_size;
                std::memcpy(c.v_term, vb.terminal, sizeof(c.v_term));
                break;
            }
            default:
                why = "spatial DIR component operator is unsupported";
                return false;
        }
        plan.comp[n++] = c;
    }
    if (!any) {
        why = "spatial DIR has no active component";
        return false;
    }
    plan.count = n;
    return true;
}

} // namespace fjb
