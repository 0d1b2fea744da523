"""Host-side grain frame plan: grain controls + film profile -> the FjVisualGrain record.

Restates the reference's Rust preparation in float32 arithmetic:

* plan: rust/film-juicer-core/src/film/grain/frame.rs:531-790 (Plan::new) -- particle
  counts per pixel, optical density per particle, fine/mid/coarse correlation
  Gaussians (radius int(4 sigma + 0.5) capped at 75), size-mix gain from the
  Gaussians' energies, per-sublayer particle tables and dye-cloud Gaussians, frame
  seeds (FNV-1a of clip, frame, session, 1), breathing constants;
* axis metadata: rust/film-juicer-core/src/film/grain.rs:78-111 (finite flags and
  16-block prefix maxima of the capture density axis);
* record packing: native/juicer_cuda_call_scope.cpp:120-160.

The descriptor hash fields are filled with non-zero identities of this module's own
making (the render path only needs them to tell equal Gaussians apart, which the
sigma/radius hash here does exactly as frame.rs:361-376 does).
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

from . import abi

F32 = np.float32
FNV_OFFSET = 0xCBF29CE484222325
FNV_PRIME = 0x100000001B3
MASK64 = (1 << 64) - 1


class PlanError(ValueError):
    def __init__(self, field_name: str, layer: int = 3, channel: int = 3):
        super().__init__(f"grain plan: {field_name} (layer {layer}, channel {channel})")
        self.field = field_name
        self.layer = layer
        self.channel = channel


def fnv_bytes(h: int, data: bytes) -> int:
    for b in data:
        h ^= b
        h = (h * FNV_PRIME) & MASK64
    return h


def fnv_u64s(values) -> int:
    h = FNV_OFFSET
    for v in values:
        h = fnv_bytes(h, struct.pack("<Q", v & MASK64))
    return h


def f32_bits(v) -> int:
    return struct.unpack("<I", struct.pack("<f", float(F32(v))))[0]


def _positive(v) -> bool:
    v = F32(v)
    return bool(np.isfinite(v) and v > 0)


def _max(a, b):  # first operand on ties / unordered, as the native std::max
    return b if a < b else a


def _min(a, b):
    return b if b < a else a


@dataclass
class Gaussian:
    sigma_px: float = 0.0
    radius: int = 0
    hash: int = 0

    @staticmethod
    def new(sigma) -> "Gaussian":
        sigma = F32(sigma)
        if not _positive(sigma):
            return Gaussian()
        expr = F32(F32(4.0) * sigma) + F32(0.5)
        if not _positive(expr):
            return Gaussian()
        radius = 75 if expr >= 75.0 else int(expr)
        if radius <= 0:
            return Gaussian()
        h = fnv_bytes(FNV_OFFSET, struct.pack("<I", f32_bits(sigma)))
        h = fnv_bytes(h, struct.pack("<i", radius))
        return Gaussian(float(sigma), radius, h)


def _round_half_away(v: float) -> float:
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def _period_rounded(value: float) -> int:
    """round() half away from zero to i64 (frame.rs:505-511)."""
    r = _round_half_away(value) if math.isfinite(value) else value
    if not math.isfinite(r) or r < -(2.0 ** 63) or r >= 2.0 ** 63:
        raise PlanError("period_frames")
    return int(r)


def _period(value: float) -> int:
    """The rounded i64 truncated to i32, at least 1."""
    i = _period_rounded(value) & 0xFFFFFFFF
    return max(i - (1 << 32) if i >= (1 << 31) else i, 1)


def _seed(clip: int, frame: int, session: int) -> int:
    h = fnv_u64s([clip, frame & MASK64, session, 1])
    return 1 if h == 0 else h


def _energy(sigma) -> float:
    g = Gaussian.new(sigma)
    if g.radius <= 0:
        return 1.0
    s2 = float(F32(sigma)) * float(F32(sigma)) * 2.0
    w = [math.exp(-(float(i - g.radius) ** 2) / s2) for i in range(2 * g.radius + 1)]
    total = 0.0
    for v in w:
        total += v
    if not (total > 0.0 and math.isfinite(total)):
        return 1.0
    inv = 1.0 / total
    sq = 0.0
    for v in w:
        n = v * inv
        sq += n * n
    e = sq * sq
    return float(F32(e if 1.0e-12 < e else 1.0e-12))


def axis_search_metadata(curves_cmy: np.ndarray, positive: bool):
    """Finite flags and 16-block prefix maxima of the density axis of each CMY channel."""
    finite = [False, False, False]
    prefix = np.zeros((3, 16), dtype=np.float32)
    if curves_cmy.shape[0] != 256:
        return finite, prefix
    for c in range(3):
        p = F32(-np.inf)
        finite[c] = True
        for i in range(256):
            a = F32(-curves_cmy[i, c]) if positive else F32(curves_cmy[i, c])
            if not np.isfinite(a):
                finite[c] = False
                break
            if p < a:
                p = a
            if i % 16 == 15:
                prefix[c, i // 16] = p
    return finite, prefix


@dataclass
class GrainInput:
    render_extent: tuple  # x, y, width, height
    full_frame_extent: tuple
    pixel_size_um: float
    frame_time: float = 0.0
    frame_rate: float = 24.0
    session_seed: int = 123
    clip_token: int = 456
    recipe_hash: int = 1
    positive: bool = False
    authored_max_cmy: tuple = (1.0, 1.0, 1.0)
    particle_area_um2: float = 0.2
    particle_scale_cmy: tuple = (0.8, 1.0, 2.0)
    particle_scale_layers: tuple = (2.5, 1.0, 0.5)
    particle_density_min_cmy: tuple = (0.07, 0.08, 0.12)
    correlation_sigma_px: float = 0.7
    dye_cloud_blur_um: float = 1.0
    sublayers_active: bool = True
    sublayer_count: int = 1
    size_mix_scale: float = 1.0
    fine_weight: float = 1.0
    mid_weight: float = 0.0
    coarse_weight: float = 0.0
    clump_morph_period_sec: float = 8.0
    layer_curves: list | None = None  # [layer][channel] -> 1-D arrays (only maxima are used)
    layers_hash: int = 12345


@dataclass
class Plan:
    frame0: int
    frame_alpha: float
    seed_base: int
    seed_base_next: int
    pitch_px: int
    breathing_period_frames: int
    clump_morph_period_frames: int
    wang_cell_mm: float
    breathing_amplitude: float
    breathing_cell_um_small: float
    breathing_cell_um_large: float
    breathing_mix: float
    breathing_drift_um_per_frame: float
    debug_scale: float
    density_max_cmy: np.ndarray
    n_particles_cmy: np.ndarray
    od_particle_cmy: np.ndarray
    density_min_layers: np.ndarray
    density_max_layers: np.ndarray
    n_particles_layers: np.ndarray
    od_particle_layers: np.ndarray
    correlation: list
    dye_cloud: list
    size_mix_weights: np.ndarray
    size_mix_gain: float
    requires_full_frame: bool
    density_layers_hash: int


def plan(inp: GrainInput) -> Plan:
    rx, ry, rw, rh = inp.render_extent
    fx, fy, fw, fh = inp.full_frame_extent
    contains = rx >= fx and ry >= fy and rx + rw <= fx + fw and ry + rh <= fy + fh
    if (inp.recipe_hash == 0 or rw <= 0 or rh <= 0 or fw <= 0 or fh <= 0 or not contains
            or not _positive(inp.pixel_size_um) or not math.isfinite(inp.frame_time)
            or not math.isfinite(inp.frame_rate) or inp.frame_rate <= 0.0):
        raise PlanError("frame_input")
    floor = math.floor(inp.frame_time)
    if floor < -(2.0 ** 63) or floor >= 2.0 ** 63:
        raise PlanError("frame_time")
    frame0 = int(floor)
    frame_alpha = float(F32(min(max(inp.frame_time - floor, 0.0), 1.0)))
    breathing_period = _period(inp.frame_rate * 2.5)
    clump_period = _period(inp.frame_rate * float(F32(inp.clump_morph_period_sec)))
    px = F32(inp.pixel_size_um)
    film_format_mm = F32(F32(px * F32(max(fw, fh))) / F32(1000.0))
    film_scale = F32(film_format_mm / F32(10.0))
    pixel_area = F32(px * px)
    if not _positive(pixel_area):
        raise PlanError("pixel_area")
    dmax = np.zeros(3, np.float32)
    npart = np.zeros(3, np.float32)
    od = np.zeros(3, np.float32)
    ratio_sum = F32(0.0)
    refs = (F32(1.10), F32(1.27), F32(2.08))
    for c in range(3):
        mx = F32(F32(inp.authored_max_cmy[c]) + F32(inp.particle_density_min_cmy[c]))
        area = F32(F32(inp.particle_area_um2) * F32(inp.particle_scale_cmy[c]))
        ref_area = F32(F32(0.335) * refs[c])
        if not _positive(mx) or not _positive(area) or not _positive(ref_area):
            raise PlanError("particle_model", channel=c)
        count = F32(pixel_area / area)
        if inp.sublayer_count > 1:
            count = F32(count / F32(inp.sublayer_count))
        if not _positive(count):
            raise PlanError("particle_count", channel=c)
        dmax[c] = mx
        npart[c] = count
        od[c] = F32(mx / count)
        ratio_sum = F32(ratio_sum + F32(area / ref_area))
    mean = F32(F32(F32(dmax[0] + dmax[1]) + dmax[2]) / F32(3.0))
    debug_scale = F32(F32(0.25) / _max(F32(1.0e-6), mean))
    fine = F32(F32(inp.correlation_sigma_px) * np.sqrt(_max(F32(ratio_sum / F32(3.0)), F32(0.0))))
    enabled = fine > 0.0 if inp.sublayers_active else fine > 0.4
    if not enabled or not np.isfinite(fine):
        fine = F32(0.0)
    sms = F32(inp.size_mix_scale)
    mixed = fine > 0.0 and sms > 1.0 and (inp.mid_weight > 0.0 or inp.coarse_weight > 0.0)
    mid = F32(0.0)
    coarse = F32(0.0)
    if mixed:
        raw = F32(fine * np.sqrt(sms))
        coarse = _max(fine, _min(raw, F32(fine * F32(4.0))))
        mid = np.sqrt(_max(F32(0.0), F32(fine * coarse)))
        mixed = _positive(mid) and _positive(coarse)
    correlation = [Gaussian.new(fine), Gaussian(), Gaussian()]
    weights = np.array([1.0, 0.0, 0.0], np.float32)
    gain = F32(1.0)
    if mixed:
        correlation[1] = Gaussian.new(mid)
        correlation[2] = Gaussian.new(coarse)
        fw_, mw_, cw_ = F32(inp.fine_weight), F32(inp.mid_weight), F32(inp.coarse_weight)
        weights = np.array([fw_, mw_, cw_], np.float32)
        fe, me, ce = F32(_energy(fine)), F32(_energy(mid)), F32(_energy(coarse))
        mid_scale = np.sqrt(sms)
        ratio_mid = F32(F32(mid_scale * me) / _max(F32(1.0e-12), fe))
        ratio_coarse = F32(F32(sms * ce) / _max(F32(1.0e-12), fe))
        den = F32(F32(F32(fw_ * fw_) + F32(F32(mw_ * mw_) * ratio_mid)) + F32(F32(cw_ * cw_) * ratio_coarse))
        if not np.isfinite(den) or den <= 1.0e-12:
            raise PlanError("size_mix")
        gain = F32(F32(1.0) / np.sqrt(den))
    dmin_l = np.zeros((3, 3), np.float32)
    dmax_l = np.zeros((3, 3), np.float32)
    n_l = np.zeros((3, 3), np.float32)
    od_l = np.zeros((3, 3), np.float32)
    dye = [[Gaussian() for _ in range(3)] for _ in range(3)]
    if inp.sublayers_active:
        maxima = np.zeros((3, 3), np.float32)
        for layer in range(3):
            for c in range(3):
                curve = np.asarray(inp.layer_curves[layer][c], dtype=np.float32)
                finite = curve[np.isfinite(curve)]
                if finite.size == 0:
                    raise PlanError("layer_curve", layer, c)
                maxima[layer, c] = F32(np.max(finite.astype(np.float64)))
        for c in range(3):
            total = F32(0.0)
            for layer in range(3):
                total = F32(total + maxima[layer, c])
            if not _positive(total):
                raise PlanError("density_layer_total", channel=c)
            for layer in range(3):
                frac = F32(maxima[layer, c] / total)
                mn = F32(frac * F32(inp.particle_density_min_cmy[c]))
                mx = F32(maxima[layer, c] + mn)
                area = F32(F32(F32(inp.particle_area_um2) * F32(inp.particle_scale_cmy[c]))
                           * F32(inp.particle_scale_layers[layer]))
                if not _positive(area):
                    raise PlanError("layer_particle_area", layer, c)
                count = F32(F32(pixel_area * frac) / area)
                if not _positive(count):
                    raise PlanError("layer_particle_count", layer, c)
                o = F32(mx / count)
                dmin_l[layer, c], dmax_l[layer, c], n_l[layer, c], od_l[layer, c] = mn, mx, count, o
                dye[layer][c] = Gaussian.new(F32(F32(inp.dye_cloud_blur_um) * np.sqrt(_max(F32(0.0), o))))
    full_needed = any(g.radius > 0 for g in correlation) or any(g.radius > 0 for row in dye for g in row)
    if full_needed and tuple(inp.render_extent) != tuple(inp.full_frame_extent):
        raise PlanError("partial_frame")
    return Plan(frame0=frame0, frame_alpha=frame_alpha,
                seed_base=_seed(inp.clip_token, frame0, inp.session_seed),
                seed_base_next=_seed(inp.clip_token, frame0 + 1, inp.session_seed),
                pitch_px=fh, breathing_period_frames=breathing_period, clump_morph_period_frames=clump_period,
                wang_cell_mm=2.0, breathing_amplitude=float(F32(0.01902219)),
                breathing_cell_um_small=float(F32(F32(2500.0) * film_scale)),
                breathing_cell_um_large=float(F32(F32(5000.0) * film_scale)),
                breathing_mix=float(F32(0.30)), breathing_drift_um_per_frame=1.0, debug_scale=float(debug_scale),
                density_max_cmy=dmax, n_particles_cmy=npart, od_particle_cmy=od, density_min_layers=dmin_l,
                density_max_layers=dmax_l, n_particles_layers=n_l, od_particle_layers=od_l,
                correlation=correlation, dye_cloud=dye, size_mix_weights=weights, size_mix_gain=float(gain),
                requires_full_frame=bool(full_needed),
                density_layers_hash=inp.layers_hash if inp.sublayers_active else 0)


@dataclass
class GrainCoefficients:
    micro_structure: tuple = (0.2, 30.0)
    clump_temporal_mix: float = 0.0
    amplitude: float = 1.0
    chroma_mix: float = 0.0
    chroma_shared_weight: float = 1.0
    chroma_independent_weight: float = 0.0
    uniformity_cmy: tuple = (0.97, 0.97, 0.99)
    debug_view: int = 0


def visual_grain_record(inp: GrainInput, p: Plan, coeff: GrainCoefficients,
                        curves_cmy: np.ndarray | None = None) -> "abi.FjVisualGrain":
    """Packs plan + recipe coefficients into the C-ABI record (curves_cmy: the capture
    density curves, N x 3, for the layer-axis search metadata)."""
    g = abi.FjVisualGrain()
    flags = abi.FJ_GRAIN_ACTIVE
    if inp.sublayers_active:
        flags |= abi.FJ_GRAIN_SUBLAYERS
    if p.requires_full_frame:
        flags |= abi.FJ_GRAIN_FULL_FRAME
    if inp.sublayers_active and curves_cmy is not None:
        finite, prefix = axis_search_metadata(np.asarray(curves_cmy, np.float32), inp.positive)
        for c in range(3):
            if finite[c]:
                flags |= abi.FJ_GRAIN_AXIS_FINITE_C << c
            for b in range(16):
                g.layer_axis_block_prefix_max[c][b] = float(prefix[c, b])
    g.flags = flags
    g.debug_view = coeff.debug_view
    for ext, src in ((g.render_extent, inp.render_extent), (g.full_frame_extent, inp.full_frame_extent)):
        ext.x, ext.y, ext.width, ext.height = src
    g.pixel_size_um = inp.pixel_size_um
    g.frame0 = p.frame0
    g.frame_alpha = p.frame_alpha
    g.seed_base = p.seed_base
    g.seed_base_next = p.seed_base_next
    g.session_seed = inp.session_seed
    g.clip_token = inp.clip_token
    g.pitch_px = p.pitch_px
    g.breathing_period_frames = p.breathing_period_frames
    g.clump_morph_period_frames = p.clump_morph_period_frames
    g.wang_cell_mm = p.wang_cell_mm
    g.breathing_amplitude = p.breathing_amplitude
    g.breathing_cell_um_small = p.breathing_cell_um_small
    g.breathing_cell_um_large = p.breathing_cell_um_large
    g.breathing_mix = p.breathing_mix
    g.breathing_drift_um_per_frame = p.breathing_drift_um_per_frame
    g.debug_scale = p.debug_scale
    for c in range(3):
        g.density_max_cmy[c] = float(p.density_max_cmy[c])
        g.n_particles_cmy[c] = float(p.n_particles_cmy[c])
        g.od_particle_cmy[c] = float(p.od_particle_cmy[c])
        g.particle_density_min_cmy[c] = float(F32(inp.particle_density_min_cmy[c]))
        g.uniformity_cmy[c] = float(F32(coeff.uniformity_cmy[c]))
        g.size_mix_weights[c] = float(p.size_mix_weights[c])
        for layer in range(3):
            g.density_min_layers[layer][c] = float(p.density_min_layers[layer, c])
            g.density_max_layers[layer][c] = float(p.density_max_layers[layer, c])
            g.n_particles_layers[layer][c] = float(p.n_particles_layers[layer, c])
            g.od_particle_layers[layer][c] = float(p.od_particle_layers[layer, c])
            d = p.dye_cloud[layer][c]
            g.dye_cloud[layer][c].sigma_px, g.dye_cloud[layer][c].radius, g.dye_cloud[layer][c].hash = \
                d.sigma_px, d.radius, d.hash
    for i in range(3):
        cg = p.correlation[i]
        g.correlation[i].sigma_px, g.correlation[i].radius, g.correlation[i].hash = cg.sigma_px, cg.radius, cg.hash
    g.size_mix_gain = p.size_mix_gain
    g.sublayer_count = inp.sublayer_count
    g.micro_structure[0], g.micro_structure[1] = coeff.micro_structure
    g.clump_temporal_mix = coeff.clump_temporal_mix
    g.size_mix_scale = inp.size_mix_scale
    g.amplitude = coeff.amplitude
    g.chroma_mix = coeff.chroma_mix
    g.chroma_shared_weight = coeff.chroma_shared_weight
    g.chroma_independent_weight = coeff.chroma_independent_weight
    g.recipe_hash = inp.recipe_hash
    g.density_layers_hash = p.density_layers_hash
    g.hash = fnv_u64s([p.seed_base, inp.recipe_hash, p.density_layers_hash, 7]) or 1
    return g


@dataclass
class Noise:
    """Static grain noise with the arrays that back the record's spans."""
    stbn: np.ndarray  # uint8 [frames][h][w]
    wang_tiles: np.ndarray  # uint8 [tile][h][w]
    wang_lut: np.ndarray  # uint8 [colors^4]
    colors: int = 2
    record: "abi.FjStaticNoise" = field(init=False)

    def __post_init__(self):
        self.stbn = np.ascontiguousarray(self.stbn, dtype=np.uint8)
        self.wang_tiles = np.ascontiguousarray(self.wang_tiles, dtype=np.uint8)
        self.wang_lut = np.ascontiguousarray(self.wang_lut, dtype=np.uint8)
        r = abi.FjStaticNoise()
        u8p = abi.C.POINTER(abi.C.c_uint8)
        r.stbn.data = self.stbn.ctypes.data_as(u8p)
        r.stbn.count = self.stbn.size
        r.stbn_frames, r.stbn_height, r.stbn_width = self.stbn.shape
        r.wang_tiles.data = self.wang_tiles.ctypes.data_as(u8p)
        r.wang_tiles.count = self.wang_tiles.size
        r.wang_tile_count, r.wang_height, r.wang_width = self.wang_tiles.shape
        r.wang_lut.data = self.wang_lut.ctypes.data_as(u8p)
        r.wang_lut.count = self.wang_lut.size
        r.wang_colors = self.colors
        self.record = r


def wang_lut_two_colors() -> np.ndarray:
    """Tile index for each (left, right, top, bottom) 2-colour edge combination,
    addressed ((L*2+R)*2+T)*2+B (data_io/noise.rs:346-374); the reference's tile set
    (Resources/Noise/Wang/tiles.json) numbers its tiles R + 2L + 4B + 8T."""
    lut = np.zeros(16, np.uint8)
    for l in range(2):
        for r in range(2):
            for t in range(2):
                for b in range(2):
                    lut[((l * 2 + r) * 2 + t) * 2 + b] = r + 2 * l + 4 * b + 8 * t
    return lut


def synthetic_noise(seed: int = 7, stbn_shape=(256, 512, 512), wang_shape=(16, 256, 256)) -> Noise:
    """Seeded uniform bytes in the production shapes (blue-noise 512x512x256, Wang
    16 tiles of 256x256, two edge colours) standing in for the resource files."""
    rng = np.random.default_rng(seed)
    return Noise(rng.integers(0, 256, size=stbn_shape, dtype=np.uint8),
                 rng.integers(0, 256, size=wang_shape, dtype=np.uint8), wang_lut_two_colors())
