// fjb_film_defects.cu -- procedural film and gate defects: dust and scratches.
//
// Restates src/Cuda/Scan/JuicerCudaScanPipeline.cu of the reference:
//   identity / lanes   :803-819, :846-883  splitmix64 hashes of (session seed, clip token
//                                           for the film families, cell x, cell y, family,
//                                           slot); attribute lanes remixed per salt;
//   candidates         :895-1136           compact dust (three ellipses), fibres and
//                                           scratches (tapered four-vertex strokes);
//   cross section      :1138-1243          union of the horizontal intervals of a
//                                           candidate at one height, weighted by depth;
//   coverage           :1245-1273          3 softness shifts x 8 rows x 3 columns;
//   family             :1275-1320          candidates of the cells that can reach a
//                                           pixel; retained *= 1 - strength * coverage;
//   film defects       :2056-2079          dust transmittance plane, scratches scale the
//                                           density planes;
//   gate mask          :2081-2094          gate dust x gate scratch at the half-resolution
//                                           gate grid (sample step x 2).
// The hashing constants, the attribute lane numbers and the floating-point expressions
// are the reference's: they define the defect pattern, which must match it bit for bit.
//
// B200 schedule. A pre-pass builds every candidate of the frame's cell range once, one
// per thread, into a particle table (a candidate depends only on its cell address). A
// CTA covers a 32 x 8 pixel tile: its threads read the candidates of the tile's cell
// range kChunk at a time from the table (or build them, when no table was given) and keep
// -- in candidate order -- only the active ones whose bounding box, widened by softness
// and the pixel footprint, can reach the tile; the tile's pixels then multiply over
// that short list. A candidate
// that cannot reach a pixel contributes exactly 1 - strength * 0 = 1 to its product, so
// the culling changes no result (candidates with a non-finite strength are kept). The
// reference makes every pixel visit every candidate of its tile.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "fjb_film_defects.h"
#include "fjb_launches.h"

namespace fjb {

namespace {

constexpr int kTileX = 32, kTileY = 8, kTileThreads = kTileX * kTileY;
// candidates a tile takes per round (the first kChunk threads read or build one each);
// the shared list of reachable candidates holds at most one round
constexpr int kChunk = 64;

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

// 24 high bits of a remixed hash as a float in [0, 1).
__device__ __forceinline__ float lane(uint64_t identity, unsigned k) {
    const uint64_t h = mix64(identity ^ (0xD6E8FEB86659FD93ULL * ((uint64_t)k + 1ULL)));
    return (float)((h >> 40) & 0xFFFFFFu) * (1.0f / 16777216.0f);
}

struct Particle {
    float cx, cy, xmin, xmax, ymin, ymax, strength, softness;
    float ex[3], ey[3], ea[3], eb[3], ec[3]; // ellipses: centre and x^2, xy, y^2 coefficients
    float px[4], py[4], width[4], depth[4];  // stroke vertices (full widths)
    int stroke, active;
};

struct Stroke {
    float length, drift, angle;
    float t[4], width[4], depth[4];
};

__device__ uint64_t particle_identity(const FjFilmEffects& e, int family, int64_t cell_x, int64_t cell_y, int slot) {
    uint64_t h = mix64(e.session_seed);
    if (family < 2) h = mix64(h ^ mix64(e.clip_token));
    h = mix64(h ^ (uint64_t)cell_x);
    h = mix64(h ^ (uint64_t)cell_y);
    h = mix64(h ^ (0x8EBC6AF09C88C6E3ULL * (uint64_t)(family + 1)));
    return mix64(h ^ (uint64_t)slot);
}

// Bulk / tail mixture of a length: t = v^3 spreads over the bulk or the tail range.
__device__ float mixture(float u, float v, float minimum, float bulk_max, float maximum, float tail_fraction) {
    const float t = v * v * v;
    return u < tail_fraction ? bulk_max + (maximum - bulk_max) * t : minimum + (bulk_max - minimum) * t;
}

__device__ void make_stroke(Particle& q, uint64_t h, const Stroke& s) {
    float dx[4] = {0.0f, (lane(h, 12) - 0.5f) * s.drift * s.length, (lane(h, 13) - 0.5f) * s.drift * s.length,
                   (lane(h, 14) - 0.5f) * s.drift * s.length};
    float total = 0.0f;
    float widest = 0.0f;
    for (int i = 1; i < 4; ++i) total += hypotf(dx[i] - dx[i - 1], s.length * (s.t[i] - s.t[i - 1]));
    for (float w : s.width) widest = fmaxf(widest, w);
    const float norm = s.length / total;
    const float c = cosf(s.angle);
    const float sn = sinf(s.angle);
    q.stroke = 1;
    q.xmin = q.ymin = 1.0e30f;
    q.xmax = q.ymax = -1.0e30f;
    for (int i = 0; i < 4; ++i) {
        const float y = (s.t[i] - 0.5f) * s.length * norm;
        const float x = dx[i] * norm;
        q.px[i] = x * c - y * sn;
        q.py[i] = x * sn + y * c;
        q.width[i] = s.width[i];
        q.depth[i] = s.depth[i];
        q.xmin = fminf(q.xmin, q.px[i] - widest * 0.5f);
        q.xmax = fmaxf(q.xmax, q.px[i] + widest * 0.5f);
        q.ymin = fminf(q.ymin, q.py[i] - widest * 0.5f);
        q.ymax = fmaxf(q.ymax, q.py[i] + widest * 0.5f);
    }
}

// Piecewise-linear opacity over the faint / intermediate / dense thirds of the draw.
__device__ float dust_opacity(const FjDust& d, bool fiber, float u) {
    const float lo = fiber ? d.fiber_opacity_min : d.compact_opacity_min;
    const float faint = fiber ? d.fiber_opacity_faint_end : d.compact_opacity_faint_end;
    const float mid = fiber ? d.fiber_opacity_intermediate_end : d.compact_opacity_intermediate_end;
    const float hi = fiber ? d.fiber_opacity_max : d.compact_opacity_max;
    const float c1 = d.opacity_faint_cumulative;
    const float c2 = d.opacity_intermediate_cumulative;
    if (u < c1) return lo + (faint - lo) * (u / c1);
    if (u < c2) return faint + (mid - faint) * ((u - c1) / (c2 - c1));
    return mid + (hi - mid) * ((u - c2) / (1.0f - c2));
}

__device__ float softness_of(float u, float lo, float hi, float cap_fraction, float size) {
    return fminf(lo + (hi - lo) * u * u, size * cap_fraction);
}

__device__ Particle make_particle(const FjFilmEffects& e, int family, int64_t cell_x, int64_t cell_y, int slot,
                                  int offset_x, int offset_y) {
    Particle q{};
    const FjDust& dust = family == 0 ? e.film_dust : e.gate_dust;
    const FjScratch& scratch = family == 1 ? e.film_scratch : e.gate_scratch;
    const bool is_dust = family == 0 || family == 2;
    const uint64_t h = particle_identity(e, family, cell_x, cell_y, slot);
    if (lane(h, 0) >= (is_dust ? dust.slot_probability : scratch.slot_probability)) return q;
    const float cw = is_dust ? dust.cell_width_mm : scratch.cell_width_mm;
    const float ch = is_dust ? dust.cell_height_mm : scratch.cell_height_mm;
    q.cx = ((float)offset_x + lane(h, 1)) * cw;
    q.cy = ((float)offset_y + lane(h, 2)) * ch;
    q.active = 1;
    if (is_dust) {
        const float angle = lane(h, 4) * 6.28318530718f;
        const bool fiber = lane(h, 5) < dust.fiber_fraction;
        q.strength = dust_opacity(dust, fiber, lane(h, 3));
        if (fiber) {
            const float length = dust.fiber_length_min_mm + (dust.fiber_length_max_mm - dust.fiber_length_min_mm) * lane(h, 6);
            const float width = dust.fiber_width_min_mm + (dust.fiber_width_max_mm - dust.fiber_width_min_mm) * lane(h, 7);
            q.softness = softness_of(lane(h, 47), dust.softness_min_mm, dust.softness_max_mm,
                                     dust.softness_size_cap_fraction, width);
            const float k1 = dust.fiber_first_knot_min + (dust.fiber_first_knot_max - dust.fiber_first_knot_min) * lane(h, 30);
            const float k2 =
                dust.fiber_second_knot_min + (dust.fiber_second_knot_max - dust.fiber_second_knot_min) * lane(h, 31);
            Stroke s{};
            s.length = length;
            s.drift = dust.fiber_drift_fraction;
            s.angle = angle;
            s.t[0] = 0.0f;
            s.t[1] = k1;
            s.t[2] = k2;
            s.t[3] = 1.0f;
            const float wspan = dust.fiber_interior_width_max_fraction - dust.fiber_interior_width_min_fraction;
            s.width[1] = width * (dust.fiber_interior_width_min_fraction + wspan * lane(h, 21));
            s.width[2] = width * (dust.fiber_interior_width_min_fraction + wspan * lane(h, 22));
            for (float& d : s.depth) d = 1.0f;
            make_stroke(q, h, s);
        } else {
            const float diameter = mixture(lane(h, 6), lane(h, 7), dust.diameter_min_mm, dust.diameter_bulk_max_mm,
                                           dust.diameter_max_mm, dust.diameter_tail_fraction);
            q.softness = softness_of(lane(h, 47), dust.softness_min_mm, dust.softness_max_mm,
                                     dust.softness_size_cap_fraction, diameter);
            float ox[3]{}, oy[3]{}, rx[3]{}, ry[3]{}, rot[3]{};
            rx[0] = 1.0f;
            ry[0] = dust.compact_dominant_aspect_min +
                    (dust.compact_dominant_aspect_max - dust.compact_dominant_aspect_min) * lane(h, 32);
            rot[0] = angle;
            const float dc = cosf(angle);
            const float ds = sinf(angle);
            float enclosing = 1.0f;
            for (int i = 1; i < 3; ++i) {
                rx[i] = dust.compact_subsidiary_scale_min +
                        (dust.compact_subsidiary_scale_max - dust.compact_subsidiary_scale_min) * lane(h, 32 + i * 5);
                const float aspect =
                    dust.compact_subsidiary_aspect_min +
                    (dust.compact_subsidiary_aspect_max - dust.compact_subsidiary_aspect_min) * lane(h, 33 + i * 5);
                ry[i] = rx[i] * aspect;
                const float polar = lane(h, 34 + i * 5) * 6.28318530718f;
                const float radial = dust.compact_subsidiary_offset_max * sqrtf(lane(h, 35 + i * 5));
                const float lx = radial * cosf(polar);
                const float ly = radial * ry[0] * sinf(polar);
                ox[i] = lx * dc - ly * ds;
                oy[i] = lx * ds + ly * dc;
                rot[i] = angle + (2.0f * lane(h, 36 + i * 5) - 1.0f) * dust.compact_subsidiary_angle_max_radians;
                enclosing = fmaxf(enclosing, hypotf(ox[i], oy[i]) + fmaxf(rx[i], ry[i]));
            }
            const float scale = diameter * 0.5f / enclosing;
            q.xmin = q.ymin = 1.0e30f;
            q.xmax = q.ymax = -1.0e30f;
            for (int i = 0; i < 3; ++i) {
                const float a = rx[i] * scale;
                const float b = ry[i] * scale;
                const float c = cosf(rot[i]);
                const float s = sinf(rot[i]);
                q.ex[i] = ox[i] * scale;
                q.ey[i] = oy[i] * scale;
                q.ea[i] = c * c / (a * a) + s * s / (b * b);
                q.eb[i] = c * s * (1.0f / (a * a) - 1.0f / (b * b));
                q.ec[i] = s * s / (a * a) + c * c / (b * b);
                const float hx = sqrtf(a * a * c * c + b * b * s * s);
                const float hy = sqrtf(a * a * s * s + b * b * c * c);
                q.xmin = fminf(q.xmin, q.ex[i] - hx);
                q.xmax = fmaxf(q.xmax, q.ex[i] + hx);
                q.ymin = fminf(q.ymin, q.ey[i] - hy);
                q.ymax = fmaxf(q.ymax, q.ey[i] + hy);
            }
        }
    } else {
        const FjScratch& sp = scratch;
        q.strength = sp.strength_min + (sp.strength_max - sp.strength_min) * lane(h, 3);
        const float length =
            mixture(lane(h, 6), lane(h, 7), sp.length_min_mm, sp.length_bulk_max_mm, sp.length_max_mm, sp.length_tail_fraction);
        const float width =
            mixture(lane(h, 8), lane(h, 9), sp.width_min_mm, sp.width_bulk_max_mm, sp.width_max_mm, sp.width_tail_fraction);
        q.softness = softness_of(lane(h, 47), sp.softness_min_mm, sp.softness_max_mm, sp.softness_size_cap_fraction, width);
        Stroke s{};
        s.length = length;
        s.drift = sp.drift_fraction;
        const bool interrupted = lane(h, 30) < sp.interruption_probability;
        if (interrupted) {
            const float centre = sp.gap_center_min + (sp.gap_center_max - sp.gap_center_min) * lane(h, 31);
            const float span = sp.gap_span_min + (sp.gap_span_max - sp.gap_span_min) * lane(h, 32);
            s.t[1] = centre - span * 0.5f;
            s.t[2] = centre + span * 0.5f;
        } else {
            s.t[1] = sp.first_knot_min + (sp.first_knot_max - sp.first_knot_min) * lane(h, 31);
            s.t[2] = sp.second_knot_min + (sp.second_knot_max - sp.second_knot_min) * lane(h, 32);
        }
        s.t[3] = 1.0f;
        for (int i = 0; i < 4; ++i) {
            const float wf = sp.interior_width_min_fraction +
                             (sp.interior_width_max_fraction - sp.interior_width_min_fraction) * lane(h, 33 + i);
            s.width[i] = (i == 1 || i == 2 || lane(h, 37 + i) < sp.endpoint_abrupt_probability) ? width * wf : 0.0f;
            s.depth[i] = sp.interior_depth_min_fraction +
                         (sp.interior_depth_max_fraction - sp.interior_depth_min_fraction) * lane(h, 41 + i);
        }
        if (interrupted) s.depth[1] = s.depth[2] = 0.0f;
        if (length <= sp.scuff_length_max_mm && lane(h, 45) < sp.scuff_probability)
            s.angle = (2.0f * lane(h, 46) - 1.0f) * sp.scuff_angle_max_radians;
        make_stroke(q, h, s);
    }
    return q;
}

// Length of the particle's cross section at height y inside [lo_x, hi_x], each piece
// weighted by its depth (the deepest where pieces overlap).
__device__ float cross_section(const Particle& q, float y, float lo_x, float hi_x) {
    float lo[5]{}, hi[5]{}, depth[5]{};
    int n = 0;
    for (int i = 0; i < 3; ++i) {
        float a = 0.0f, b = 0.0f;
        if (!q.stroke) {
            const float dy = y - q.ey[i];
            const float disc = q.ea[i] - (q.ea[i] * q.ec[i] - q.eb[i] * q.eb[i]) * dy * dy;
            if (disc <= 0.0f) continue;
            const float centre = q.ex[i] - q.eb[i] * dy / q.ea[i];
            const float half = sqrtf(disc) / q.ea[i];
            a = centre - half;
            b = centre + half;
        } else {
            // the tapered quadrilateral of segment i
            const float dx = q.px[i + 1] - q.px[i];
            const float dy = q.py[i + 1] - q.py[i];
            const float inv = rsqrtf(dx * dx + dy * dy);
            const float nx = -dy * inv * 0.5f;
            const float ny = dx * inv * 0.5f;
            const float vx[4] = {q.px[i] + nx * q.width[i], q.px[i + 1] + nx * q.width[i + 1],
                                 q.px[i + 1] - nx * q.width[i + 1], q.px[i] - nx * q.width[i]};
            const float vy[4] = {q.py[i] + ny * q.width[i], q.py[i + 1] + ny * q.width[i + 1],
                                 q.py[i + 1] - ny * q.width[i + 1], q.py[i] - ny * q.width[i]};
            a = 1.0e30f;
            b = -1.0e30f;
            for (int k = 0; k < 4; ++k) {
                const int k1 = (k + 1) % 4;
                if (y >= fminf(vy[k], vy[k1]) && y < fmaxf(vy[k], vy[k1])) {
                    const float x = vx[k] + (y - vy[k]) / (vy[k1] - vy[k]) * (vx[k1] - vx[k]);
                    a = fminf(a, x);
                    b = fmaxf(b, x);
                }
            }
        }
        a = fmaxf(lo_x, a);
        b = fminf(hi_x, b);
        if (b > a) {
            depth[n] = 1.0f;
            if (q.stroke) {
                const float dx = q.px[i + 1] - q.px[i];
                const float dy = q.py[i + 1] - q.py[i];
                const float mid = 0.5f * (a + b);
                const float den = dx * dx + dy * dy;
                const float t = fminf(1.0f, fmaxf(0.0f, ((mid - q.px[i]) * dx + (y - q.py[i]) * dy) / den));
                depth[n] = q.depth[i] + (q.depth[i + 1] - q.depth[i]) * t;
            }
            lo[n] = a;
            hi[n] = b;
            ++n;
        }
    }
    if (q.stroke) {
        // round joints at the two interior vertices
        for (int i = 1; i < 3; ++i) {
            const float r = q.width[i] * 0.5f;
            const float dy = y - q.py[i];
            if (fabsf(dy) >= r) continue;
            const float chord = sqrtf(fmaxf(0.0f, r * r - dy * dy));
            const float a = fmaxf(lo_x, q.px[i] - chord);
            const float b = fminf(hi_x, q.px[i] + chord);
            if (b > a) {
                lo[n] = a;
                hi[n] = b;
                depth[n] = q.depth[i];
                ++n;
            }
        }
    }
    float ends[10]{};
    for (int i = 0; i < n; ++i) {
        ends[2 * i] = lo[i];
        ends[2 * i + 1] = hi[i];
    }
    for (int i = 1; i < 2 * n; ++i)
        for (int j = i; j > 0 && ends[j] < ends[j - 1]; --j) {
            const float v = ends[j];
            ends[j] = ends[j - 1];
            ends[j - 1] = v;
        }
    float length = 0.0f;
    for (int i = 1; i < 2 * n; ++i) {
        const float mid = (ends[i - 1] + ends[i]) * 0.5f;
        float strength = 0.0f;
        for (int k = 0; k < n; ++k)
            if (mid >= lo[k] && mid <= hi[k]) strength = fmaxf(strength, depth[k]);
        length += (ends[i] - ends[i - 1]) * strength;
    }
    return length;
}

// Fraction of the pixel footprint (sx x sy mm at x, y) the particle covers, with its
// softness as a 3 x 3 box of shifts.
__device__ float coverage(const Particle& q, float x, float y, float sx, float sy) {
    x -= q.cx;
    y -= q.cy;
    if (x + sx * 0.5f + q.softness < q.xmin || x - sx * 0.5f - q.softness > q.xmax ||
        y + sy * 0.5f + q.softness < q.ymin || y - sy * 0.5f - q.softness > q.ymax)
        return 0.0f;
    float area = 0.0f;
    for (int soft = 0; soft < 3; ++soft) {
        const float shift = ((float)soft - 1.0f) * q.softness;
        const float bottom = fmaxf(q.ymin, y - sy * 0.5f + shift);
        const float top = fminf(q.ymax, y + sy * 0.5f + shift);
        if (!(top > bottom)) continue;
        float sum = 0.0f;
        for (int row = 0; row < 8; ++row) {
            const float yy = bottom + ((float)row + 0.5f) * (top - bottom) / 8.0f;
            for (int col = 0; col < 3; ++col) {
                const float off = ((float)col - 1.0f) * q.softness;
                sum += cross_section(q, yy, x - sx * 0.5f + off, x + sx * 0.5f + off);
            }
        }
        area += sum * (top - bottom) / 72.0f;
    }
    return fminf(1.0f, fmaxf(0.0f, area / (sx * sy)));
}

// Particles of one family built once per frame: the candidates of cells [x0, x0 +
// columns) x [y0, y0 + rows) (relative to the family's origin), two slots per cell, at
// index ((y - y0) * columns + (x - x0)) * 2 + slot. A particle depends only on its cell
// address, so a tile reads it instead of building it again. p == nullptr: tiles build
// their candidates themselves.
struct ParticleTable {
    const Particle* p;
    int x0, y0, columns, rows;
};

struct FrameTables {
    ParticleTable t[2];
};

__global__ void __launch_bounds__(256) build_particles_kernel(const __grid_constant__ FjFilmEffects e, int family,
                                                              int x0, int y0, int columns, int rows, Particle* out) {
    const long long total = (long long)columns * rows * 2;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= total) return;
    const int dx = x0 + (int)((o / 2) % columns);
    const int dy = y0 + (int)((o / 2) / columns);
    out[o] = make_particle(e, family, e.origins[family].cell_x + dx, e.origins[family].cell_y + dy, (int)(o % 2), dx, dy);
}

// One family at the pixels of a tile: `tile` is the tile's first pixel in the family's
// pixel grid, (px, py) this thread's pixel there, `scale` the grid's step in sample
// steps. Returns the retained fraction (1 when the family is off).
__device__ float family_retained(const FjFilmEffects& e, int family, int tile_x, int tile_y, int px, int py, float scale,
                                 const ParticleTable& table, Particle* list, int* counts) {
    const bool is_dust = family == 0 || family == 2;
    const FjDust& dp = family == 0 ? e.film_dust : e.gate_dust;
    const FjScratch& sp = family == 1 ? e.film_scratch : e.gate_scratch;
    const float probability = is_dust ? dp.slot_probability : sp.slot_probability;
    if (!(probability > 0.0f)) return 1.0f;
    const float cw = is_dust ? dp.cell_width_mm : sp.cell_width_mm;
    const float ch = is_dust ? dp.cell_height_mm : sp.cell_height_mm;
    const float support_x = is_dust ? dp.support_x_mm + dp.softness_max_mm : sp.support_x_mm + sp.softness_max_mm;
    const float support_y = is_dust ? dp.support_y_mm + dp.softness_max_mm : sp.support_y_mm + sp.softness_max_mm;
    const FjDefectOrigin& origin = e.origins[family];
    const float step_x = e.sample_step_x_mm * scale;
    const float step_y = e.sample_step_y_mm * scale;
    const float base_x = origin.local_x_mm;
    const float base_y = origin.local_y_mm;
    const int x0 = (int)floorf((base_x + (float)tile_x * step_x - support_x) / cw);
    const int y0 = (int)floorf((base_y + (float)tile_y * step_y - support_y) / ch);
    const int x1 = (int)floorf((base_x + (float)(tile_x + kTileX) * step_x + support_x) / cw);
    const int y1 = (int)floorf((base_y + (float)(tile_y + kTileY) * step_y + support_y) / ch);
    const int columns = x1 - x0 + 1;
    const int total = columns * (y1 - y0 + 1) * 2;
    const float x = base_x + ((float)px + 0.5f) * step_x;
    const float y = base_y + ((float)py + 0.5f) * step_y;
    // the tile's extreme pixel positions, for the conservative reach test
    const float tx_lo = base_x + ((float)tile_x + 0.5f) * step_x;
    const float tx_hi = base_x + ((float)(tile_x + kTileX - 1) + 0.5f) * step_x;
    const float ty_lo = base_y + ((float)tile_y + 0.5f) * step_y;
    const float ty_hi = base_y + ((float)(tile_y + kTileY - 1) + 0.5f) * step_y;
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane_id = t & 31, warp = t >> 5;
    float retained = 1.0f;
    for (int first = 0; first < total; first += kChunk) {
        const int ordinal = first + t;
        bool keep = false;
        Particle q;
        if (t < kChunk && ordinal < total) {
            const int dx = x0 + (ordinal / 2) % columns;
            const int dy = y0 + (ordinal / 2) / columns;
            const int gx = dx - table.x0, gy = dy - table.y0;
            if (table.p && gx >= 0 && gx < table.columns && gy >= 0 && gy < table.rows) {
                const Particle* src = table.p + ((size_t)gy * table.columns + gx) * 2 + (ordinal % 2);
                q.active = src->active;
                if (q.active) q = *src;
            } else {
                q = make_particle(e, family, origin.cell_x + dx, origin.cell_y + dy, ordinal % 2, dx, dy);
            }
            if (q.active) {
                // the per-pixel early-out of coverage(), at the tile's extreme pixels: each
                // side is monotone in the pixel position, so a side that holds there holds
                // for every pixel of the tile
                const float xl = tx_lo - q.cx, xh = tx_hi - q.cx, yl = ty_lo - q.cy, yh = ty_hi - q.cy;
                const bool away = xh + step_x * 0.5f + q.softness < q.xmin || xl - step_x * 0.5f - q.softness > q.xmax ||
                                  yh + step_y * 0.5f + q.softness < q.ymin || yl - step_y * 0.5f - q.softness > q.ymax;
                keep = !away || !isfinite(q.strength);
            }
        }
        // order-preserving compaction of the kept candidates
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        if (lane_id == 0 && warp < kChunk / 32) counts[warp] = __popc(ballot);
        __syncthreads();
        int before = 0, kept = 0;
        for (int w = 0; w < kChunk / 32; ++w) {
            before += w < warp ? counts[w] : 0;
            kept += counts[w];
        }
        if (keep) list[before + __popc(ballot & ((1u << lane_id) - 1u))] = q;
        __syncthreads();
        for (int i = 0; i < kept; ++i) retained *= 1.0f - list[i].strength * coverage(list[i], x, y, step_x, step_y);
        __syncthreads();
    }
    return retained;
}

__global__ void __launch_bounds__(kTileThreads, 3) film_defects_kernel(const __grid_constant__ FjFilmEffects e, int width,
                                                                    int height, float* c, float* m, float* yp,
                                                                    float* dust_out, FrameTables tables) {
    __shared__ Particle list[kChunk];
    __shared__ int counts[kChunk / 32];
    const int tx = blockIdx.x * kTileX, ty = blockIdx.y * kTileY;
    const int x = tx + threadIdx.x, y = ty + threadIdx.y;
    const int fx = x + e.roi_offset_x, fy = y + e.roi_offset_y;
    const int tfx = tx + e.roi_offset_x, tfy = ty + e.roi_offset_y;
    const float dust = family_retained(e, 0, tfx, tfy, fx, fy, 1.0f, tables.t[0], list, counts);
    const float retained = family_retained(e, 1, tfx, tfy, fx, fy, 1.0f, tables.t[1], list, counts);
    if (x < width && y < height) {
        const size_t i = (size_t)y * width + x;
        if (dust_out) dust_out[i] = dust;
        if (e.film_scratch.slot_probability > 0.0f) {
            c[i] *= retained;
            m[i] *= retained;
            yp[i] *= retained;
        }
    }
}

__global__ void __launch_bounds__(kTileThreads) gate_mask_kernel(const __grid_constant__ FjFilmEffects e, float* mask,
                                                                 int width, int height, FrameTables tables) {
    __shared__ Particle list[kChunk];
    __shared__ int counts[kChunk / 32];
    const int tx = blockIdx.x * kTileX, ty = blockIdx.y * kTileY;
    const int x = tx + threadIdx.x, y = ty + threadIdx.y;
    const float dust = family_retained(e, 2, tx, ty, x, y, 2.0f, tables.t[0], list, counts);
    const float scratch = family_retained(e, 3, tx, ty, x, y, 2.0f, tables.t[1], list, counts);
    if (x < width && y < height) mask[(size_t)y * width + x] = dust * scratch;
}

// Cells a family's tiles can visit over a grid of tiles whose first pixels run from
// (tx0, ty0) to (tx1, ty1), with one cell of margin on each side (the host's rounding
// may differ from the device's by an ulp); false when the family is off or its table
// would exceed kMaxTableParticles (its tiles then build their own candidates).
constexpr long long kMaxTableParticles = 1 << 18;

struct Grid {
    int x0 = 0, y0 = 0, columns = 0, rows = 0;
    size_t particles() const { return (size_t)columns * rows * 2; }
};

bool family_grid(const FjFilmEffects& e, int family, long long tx0, long long ty0, long long tx1, long long ty1,
                 float scale, Grid& g) {
    const bool is_dust = family == 0 || family == 2;
    const FjDust& dp = family == 0 ? e.film_dust : e.gate_dust;
    const FjScratch& sp = family == 1 ? e.film_scratch : e.gate_scratch;
    if (!((is_dust ? dp.slot_probability : sp.slot_probability) > 0.0f)) return false;
    const double cw = is_dust ? dp.cell_width_mm : sp.cell_width_mm;
    const double ch = is_dust ? dp.cell_height_mm : sp.cell_height_mm;
    const double sx = is_dust ? (double)dp.support_x_mm + dp.softness_max_mm : (double)sp.support_x_mm + sp.softness_max_mm;
    const double sy = is_dust ? (double)dp.support_y_mm + dp.softness_max_mm : (double)sp.support_y_mm + sp.softness_max_mm;
    const double stx = (double)e.sample_step_x_mm * scale, sty = (double)e.sample_step_y_mm * scale;
    const double bx = e.origins[family].local_x_mm, by = e.origins[family].local_y_mm;
    const double x0 = std::floor((bx + (double)tx0 * stx - sx) / cw) - 1.0;
    const double y0 = std::floor((by + (double)ty0 * sty - sy) / ch) - 1.0;
    const double x1 = std::floor((bx + (double)(tx1 + kTileX) * stx + sx) / cw) + 1.0;
    const double y1 = std::floor((by + (double)(ty1 + kTileY) * sty + sy) / ch) + 1.0;
    if (!(x0 > -2.0e9 && y0 > -2.0e9 && x1 < 2.0e9 && y1 < 2.0e9)) return false;
    const double n = (x1 - x0 + 1.0) * (y1 - y0 + 1.0) * 2.0;
    if (!(n >= 2.0 && n <= (double)kMaxTableParticles)) return false;
    g.x0 = (int)x0;
    g.y0 = (int)y0;
    g.columns = (int)(x1 - x0 + 1.0);
    g.rows = (int)(y1 - y0 + 1.0);
    return true;
}

// The two families' grids of a launch (film: families 0, 1 at the ROI-offset pixels;
// gate: families 2, 3 at the gate grid, twice the step).
void launch_grids(const FjFilmEffects& e, bool gate, int width, int height, Grid g[2], bool on[2]) {
    const long long ox = gate ? 0 : e.roi_offset_x, oy = gate ? 0 : e.roi_offset_y;
    const long long tx1 = ox + (long long)((width - 1) / kTileX) * kTileX;
    const long long ty1 = oy + (long long)((height - 1) / kTileY) * kTileY;
    for (int k = 0; k < 2; ++k) on[k] = family_grid(e, (gate ? 2 : 0) + k, ox, oy, tx1, ty1, gate ? 2.0f : 1.0f, g[k]);
}

size_t table_bytes_of(const Grid g[2], const bool on[2]) {
    size_t n = 0;
    for (int k = 0; k < 2; ++k)
        if (on[k]) n += (g[k].particles() * sizeof(Particle) + 255) / 256 * 256;
    return n;
}

// Builds the tables that fit `table` (table_bytes bytes, may be null) and returns the
// kernels' view of them.
cudaError_t build_tables(const FjFilmEffects& e, bool gate, int width, int height, void* table, size_t table_bytes,
                         FrameTables& tables, cudaStream_t stream) {
    tables = FrameTables{};
    Grid g[2];
    bool on[2];
    launch_grids(e, gate, width, height, g, on);
    if (!table || table_bytes < table_bytes_of(g, on)) return cudaSuccess;
    char* base = static_cast<char*>(table);
    for (int k = 0; k < 2; ++k) {
        if (!on[k]) continue;
        Particle* out = reinterpret_cast<Particle*>(base);
        const long long n = (long long)g[k].particles();
        fjb::count_launch();
        build_particles_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(e, (gate ? 2 : 0) + k, g[k].x0, g[k].y0,
                                                                               g[k].columns, g[k].rows, out);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
        tables.t[k] = ParticleTable{out, g[k].x0, g[k].y0, g[k].columns, g[k].rows};
        base += (g[k].particles() * sizeof(Particle) + 255) / 256 * 256;
    }
    return cudaSuccess;
}

} // namespace

size_t film_defects_table_bytes(const FjFilmEffects& e, int width, int height) {
    if (width <= 0 || height <= 0) return 0;
    Grid g[2];
    bool on[2];
    launch_grids(e, false, width, height, g, on);
    return table_bytes_of(g, on);
}

size_t gate_mask_table_bytes(const FjFilmEffects& e, int width, int height) {
    if (width <= 0 || height <= 0) return 0;
    Grid g[2];
    bool on[2];
    launch_grids(e, true, width, height, g, on);
    return table_bytes_of(g, on);
}

cudaError_t launch_film_defects(const FjFilmEffects& e, int width, int height, float* c, float* m, float* y,
                                float* dust_out, cudaStream_t stream, void* table, size_t table_bytes) {
    if (width <= 0 || height <= 0) return cudaSuccess;
    if (e.film_dust.slot_probability > 0.0f && !dust_out) return cudaErrorInvalidValue;
    FrameTables tables;
    cudaError_t err = build_tables(e, false, width, height, table, table_bytes, tables, stream);
    if (err != cudaSuccess) return err;
    fjb::count_launch();
    film_defects_kernel<<<dim3((width + kTileX - 1) / kTileX, (height + kTileY - 1) / kTileY), dim3(kTileX, kTileY), 0,
                          stream>>>(e, width, height, c, m, y, dust_out, tables);
    return cudaGetLastError();
}

cudaError_t launch_gate_mask(const FjFilmEffects& e, float* mask, int width, int height, cudaStream_t stream,
                             void* table, size_t table_bytes) {
    if (!mask || width <= 0 || height <= 0) return cudaErrorInvalidValue;
    FrameTables tables;
    cudaError_t err = build_tables(e, true, width, height, table, table_bytes, tables, stream);
    if (err != cudaSuccess) return err;
    fjb::count_launch();
    gate_mask_kernel<<<dim3((width + kTileX - 1) / kTileX, (height + kTileY - 1) / kTileY), dim3(kTileX, kTileY), 0,
                       stream>>>(e, mask, width, height, tables);
    return cudaGetLastError();
}

} // namespace fjb
