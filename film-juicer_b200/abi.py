"""ctypes mirror of include/juicer_cuda_api.h and include/juicer_b200.h.

The record layouts follow the reference boundary native/juicer_cuda_api.h:33-784
field for field (the Rust host binds the same layout through
rust/film-juicer-plugin/src/cuda/sys.rs:1712-1749). tests/test_abi_layout.py checks
these Python descriptions against the C compiler's own sizeof/offsetof.
"""
from __future__ import annotations

import ctypes as C

u32 = C.c_uint32
i32 = C.c_int32
u64 = C.c_uint64
i64 = C.c_int64
f32 = C.c_float
f64 = C.c_double
size_t = C.c_size_t
uptr = C.c_size_t  # uintptr_t
ptrdiff = C.c_ssize_t

FJ_STATUS_SUCCESS = 0
FJ_STATUS_CANCELLED = 1
FJ_STATUS_UNSUPPORTED_INPUT = 2
FJ_STATUS_PREPARATION_FAILURE = 3
FJ_STATUS_ALLOCATION_FAILURE = 4
FJ_STATUS_CUDA_FAILURE = 5
FJ_STATUS_CUFFT_FAILURE = 6
FJ_STATUS_CONTEXT_LOSS = 7
FJ_STATUS_INTERNAL_FAILURE = 8

FJ_RENDER_DEFERRED_DIR_ERROR = 1
FJ_COMPONENTS_RGB = 3
FJ_COMPONENTS_RGBA = 4
FJ_DEPTH_FLOAT32 = 1
FJ_FRAME_STREAM_PRESENT = 1
FJ_ABORT_CONTINUE = 0
FJ_ABORT_REQUESTED = 1

FJ_ROUTE_NEGATIVE_DIRECT = 0
FJ_ROUTE_NEGATIVE_PRINT = 1
FJ_ROUTE_POSITIVE_DIRECT = 2
FJ_ROUTE_POSITIVE_PRINT = 3
FJ_POLARITY_NEGATIVE = 0
FJ_POLARITY_POSITIVE = 1
FJ_RAW_HANATOS_2025 = 0
FJ_RAW_MALLETT_2019 = 1
FJ_RAW_ARCTIC_2026_BETA04 = 2
FJ_INPUT_DWG = 0
FJ_INPUT_BT2020 = 1
FJ_INPUT_ACES2065_1 = 2
FJ_INPUT_SRGB_REC709 = 3
FJ_FILM_DECODE_CCTF = 1
FJ_FILM_ADAPT_INPUT = 2
FJ_FILM_AUTO_EXPOSURE = 4
FJ_METER_CENTER_WEIGHTED = 0
FJ_METER_AVERAGE = 1
FJ_METER_MEDIAN = 2
FJ_DIR_INACTIVE = 0
FJ_DIR_NEGATIVE_DONOR_LANGMUIR = 1
FJ_DIR_POSITIVE_RECEIVER_LANGMUIR = 2
FJ_CORRECTION_ACTIVE = 1
FJ_POST_GLARE = 1
FJ_OUTPUT_SRGB = 0
FJ_COLOR_ENCODE_CCTF = 1
FJ_COLOR_INPUT_IS_OUTPUT_SPACE = 2
FJ_COLOR_GAMUT_COMPRESSION = 4
FJ_OUTPUT_ENCODING_SCHEMA = 1
FJ_CCTF_LINEAR = 0
FJ_CCTF_GAMMA = 1
FJ_CCTF_SRGB = 2
FJ_CCTF_BT2020 = 3
FJ_CCTF_PROPHOTO = 4
FJ_CCTF_DWG_INTERMEDIATE = 5
FJ_PRINT_PREFLASH = 1
FJ_OPTICS_CAMERA_DIFFUSION = 1
FJ_OPTICS_ENLARGER_DIFFUSION = 2
FJ_OPTICS_SCATTER_HALATION = 4
FJ_OPTICS_HIGHLIGHT_BOOST = 8
FJ_EFFECTS_WEAVE = 1
FJ_EFFECTS_FILM = 2
FJ_EFFECTS_GATE_TRANSMITTANCE = 4
FJ_EFFECTS_GATE_OUTPUT = 8
FJ_EFFECTS_FULL_FRAME = 16
FJ_HALATION_IDENTITY = 0
FJ_HALATION_FIR_REFLECT = 1
FJ_HALATION_YVV_REPLICATE = 2
FJ_HALATION_YVV_REPLICATE_FACTORED = 3
FJ_HALATION_TAIL_COMPONENTS = 3
FJ_HALATION_MAX_BOUNCES = 5
FJ_DIR_OPERATOR_NONE = 0
FJ_DIR_OPERATOR_IDENTITY = 1
FJ_DIR_OPERATOR_FIR_REFLECT = 2
FJ_DIR_OPERATOR_YVV_REFLECT = 3
FJ_GRAIN_ACTIVE = 1
FJ_GRAIN_SUBLAYERS = 2
FJ_GRAIN_FULL_FRAME = 4
FJ_GRAIN_AXIS_FINITE_C = 8
FJ_GRAIN_DEBUG_OFF = 0
FJ_GRAIN_DEBUG_MEAN_DENSITY = 6


def _s(name, fields):
    return type(name, (C.Structure,), {"_fields_": fields})


FjStatus = _s("FjStatus", [("category", u32), ("api", u32), ("native_code", i32)])
FjRenderOutcome = _s("FjRenderOutcome", [("status", FjStatus), ("flags", u32)])
FjErrorBuffer = _s("FjErrorBuffer", [("data", C.c_char_p), ("capacity", size_t), ("length", size_t)])
FjStringView = _s("FjStringView", [("data", C.c_char_p), ("count", size_t)])
FjFloatSpan = _s("FjFloatSpan", [("data", C.POINTER(f32)), ("count", size_t)])
FjByteSpan = _s("FjByteSpan", [("data", C.POINTER(C.c_uint8)), ("count", size_t)])
FjCudaContext = _s("FjCudaContext", [("device_id", i32), ("context", uptr)])
FjRect = _s("FjRect", [("x1", i32), ("y1", i32), ("x2", i32), ("y2", i32)])
FjExtent = _s("FjExtent", [("x", i32), ("y", i32), ("width", i32), ("height", i32)])
FjImage = _s("FjImage", [("address", uptr), ("bounds", FjRect), ("row_bytes", ptrdiff),
                         ("components", u32), ("depth", u32)])
FjEffectsGeometry = _s("FjEffectsGeometry", [("pixel_definition", FjExtent), ("canonical_x", f64),
                                             ("canonical_y", f64), ("canonical_width", f64),
                                             ("canonical_height", f64), ("scale_x", f64), ("scale_y", f64),
                                             ("pixel_aspect_ratio", f64)])
FjFrame = _s("FjFrame", [("source", FjImage), ("destination", FjImage), ("render_window", FjRect),
                         ("full_frame_extent", FjRect), ("stream", uptr), ("flags", u32),
                         ("pixel_size_um", f32), ("time_frames", f64), ("frame_rate", f64),
                         ("session_seed", u64), ("clip_token", u64), ("effects_geometry", FjEffectsGeometry)])
FjSubmission = _s("FjSubmission", [("instance_token", u64), ("frame_token", u64), ("submission_id", u64),
                                   ("upload_core_hash", u64), ("dir_hash", u64), ("scanner_hash", u64),
                                   ("auto_exposure_hash", u64)])
FjAbortQuery = C.CFUNCTYPE(u32, C.c_void_p)
FjAbortCallback = _s("FjAbortCallback", [("query", FjAbortQuery), ("user", C.c_void_p)])
FjAutoExposure = _s("FjAutoExposure", [("source_bounds", FjRect), ("meter_bounds", FjRect),
                                       ("preview_width", i32), ("preview_height", i32), ("method", u32),
                                       ("hash", u64)])
FjFilmExposure = _s("FjFilmExposure", [
    ("input_color_space", u32), ("method", u32), ("flags", u32), ("manual_exposure_ev", f32),
    ("route_correction_scale", f32), ("mallett_green_midgray_scale", f32), ("input_rgb_to_xyz", f32 * 9),
    ("input_xyz_adapt", f32 * 9), ("xyz_to_linear_srgb", f32 * 9), ("sensitivity_rgb", FjFloatSpan),
    ("tc_lut_rgba", FjFloatSpan), ("mallett_illuminant", FjFloatSpan), ("mallett_basis", FjFloatSpan),
    ("sensitivity_hash", u64), ("tc_lut_hash", u64), ("hash", u64)])
FjFilmDevelopment = _s("FjFilmDevelopment", [
    ("log_exposure", FjFloatSpan), ("density_rgb", FjFloatSpan), ("density_layers", (FjFloatSpan * 3) * 3),
    ("gamma_rgb", f32 * 3), ("density_curves_hash", u64), ("density_layers_hash", u64), ("hash", u64)])
FjDirCouplers = _s("FjDirCouplers", [
    ("mode", u32), ("matrix_rgb", f32 * 9), ("density_max_rgb", f32 * 3), ("density_ref_rgb", f32 * 3),
    ("donor_k_rgb", f32 * 3), ("receiver_c_ref_rgb", f32 * 3), ("receiver_kr_rgb", f32 * 3),
    ("compensated_axes_rgb", FjFloatSpan * 3), ("compensated_axes_hash", u64), ("hash", u64)])
FjDensityBounds = _s("FjDensityBounds", [("min_cmy", f32 * 3), ("inv_span_cmy", f32 * 3), ("hash", u64)])
FjScannerSpectra = _s("FjScannerSpectra", [
    ("dye_y", FjFloatSpan), ("dye_m", FjFloatSpan), ("dye_c", FjFloatSpan), ("weighted_x", FjFloatSpan),
    ("weighted_y", FjFloatSpan), ("weighted_z", FjFloatSpan), ("base_density", FjFloatSpan),
    ("inverse_y_normalization", f32)])
FjScannerLut = _s("FjScannerLut", [("density_bounds_hash", u64), ("resolution", u32), ("hash", u64)])
FjScannerCorrection = _s("FjScannerCorrection", [("flags", u32), ("xyz_slope", f32), ("xyz_offset", f32),
                                                 ("exposure_scale", f32)])
FjScannerPostEffects = _s("FjScannerPostEffects", [
    ("flags", u32), ("glare_percent", f32), ("glare_roughness", f32), ("glare_blur_sigma_px", f32),
    ("glare_blur_radius", i32), ("lens_blur_sigma_px", f32), ("lens_blur_radius", i32),
    ("unsharp_sigma_px", f32), ("unsharp_radius", i32), ("unsharp_amount", f32), ("hash", u64)])
FjOutputEncoding = _s("FjOutputEncoding", [
    ("schema", u32), ("cctf_kind", u32), ("gamma", f32), ("a", f32), ("b", f32), ("c", f32), ("d", f32),
    ("linear_cutoff", f32), ("dwg_to_output", f32 * 9)])
FjOutputColor = _s("FjOutputColor", [
    ("cat02", f32 * 9), ("xyz_to_rgb", f32 * 9), ("illuminant_xyz", f32 * 3), ("color_space", u32),
    ("flags", u32), ("native_rgb_to_d65_xyz", f32 * 9), ("d65_xyz_to_native_rgb", f32 * 9),
    ("lightness_knee", f32 * 3), ("chroma_knee", f32 * 3), ("gamut_cmax", FjFloatSpan),
    ("gamut_table_hash", u64), ("gamut_recipe_hash", u64), ("encoding", FjOutputEncoding)])
FjPrint = _s("FjPrint", [
    ("film_density_cmy", FjFloatSpan), ("film_base_density", FjFloatSpan), ("sensitivity_cmy", FjFloatSpan),
    ("log_exposure", FjFloatSpan), ("density_cmy", FjFloatSpan), ("main_illuminant", FjFloatSpan),
    ("preflash_illuminant", FjFloatSpan), ("flags", u32), ("main_cc_cmy", f32 * 3),
    ("preflash_cc_cmy", f32 * 3), ("exposure", f32), ("preflash_exposure", f32), ("preflash_raw_cmy", f32 * 3),
    ("normalizer", f32), ("film_density_hash", u64), ("profile_tables_hash", u64),
    ("main_illuminant_hash", u64), ("preflash_illuminant_hash", u64), ("preflash_raw_hash", u64),
    ("balance_hash", u64), ("hash", u64)])
FjDiffusion = _s("FjDiffusion", [
    ("family", u32), ("scatter_fraction", f64), ("group_weights", f64 * 3), ("group_lambda_um", f64 * 3),
    ("warmth", f64), ("spatial_scale", f64), ("pixel_size_um", f64), ("radius_px", i32),
    ("sample_hash", u64), ("hash", u64)])
FjHalationGaussian = _s("FjHalationGaussian", [("kind", u32), ("radius", i32), ("fir_weights", f32 * 19),
                                               ("yvv", f32 * 4)])
FjHalationChannel = _s("FjHalationChannel", [
    ("core", FjHalationGaussian), ("tail", FjHalationGaussian * 3), ("bounce", FjHalationGaussian * 5),
    ("total_strength", f32), ("tail_weight", f32)])
FjScatterHalation = _s("FjScatterHalation", [
    ("recipe_hash", u64), ("scatter_amount", f32), ("bounce_count", u32), ("bounce_weights", f32 * 5),
    ("renormalize", u32), ("channels", FjHalationChannel * 3)])
FjHighlightBoost = _s("FjHighlightBoost", [("recipe_hash", u64), ("protection", f64), ("sharpness", f64),
                                           ("peak_gain", f64)])
FjOptics = _s("FjOptics", [
    ("flags", u32), ("full_frame", FjExtent), ("camera", FjDiffusion), ("enlarger", FjDiffusion),
    ("diffusion_hash", u64), ("scatter_halation", FjScatterHalation), ("highlight_boost", FjHighlightBoost)])
FjDirGaussian = _s("FjDirGaussian", [
    ("sigma_px", f32), ("weight", f32), ("radius", i32), ("reference_operator", u32), ("feedforward", f64),
    ("feedback", f64 * 3), ("normalization_denominator", f64), ("feedforward_numerator", f64),
    ("feedback_numerators", f64 * 3), ("boundary_truncation_accuracy", f64),
    ("boundary_certification_tolerance", f64), ("boundary_derivation_version", u32)])
FjSpatialDir = _s("FjSpatialDir", [
    ("render_extent", FjExtent), ("full_frame_extent", FjExtent), ("filter_domain_extent", FjExtent),
    ("component_count", size_t), ("components", FjDirGaussian * 4), ("recipe_hash", u64), ("hash", u64)])
FjGrainGaussian = _s("FjGrainGaussian", [("sigma_px", f32), ("radius", i32), ("hash", u64)])
FjVisualGrain = _s("FjVisualGrain", [
    ("flags", u32), ("debug_view", u32), ("render_extent", FjExtent), ("full_frame_extent", FjExtent),
    ("pixel_size_um", f32), ("frame0", i64), ("frame_alpha", f32), ("seed_base", u64), ("seed_base_next", u64),
    ("session_seed", u64), ("clip_token", u64), ("pitch_px", i32), ("breathing_period_frames", i32),
    ("clump_morph_period_frames", i32), ("wang_cell_mm", f32), ("breathing_amplitude", f32),
    ("breathing_cell_um_small", f32), ("breathing_cell_um_large", f32), ("breathing_mix", f32),
    ("breathing_drift_um_per_frame", f32), ("debug_scale", f32), ("density_max_cmy", f32 * 3),
    ("n_particles_cmy", f32 * 3), ("od_particle_cmy", f32 * 3), ("density_min_layers", (f32 * 3) * 3),
    ("density_max_layers", (f32 * 3) * 3), ("n_particles_layers", (f32 * 3) * 3),
    ("od_particle_layers", (f32 * 3) * 3), ("correlation", FjGrainGaussian * 3),
    ("dye_cloud", (FjGrainGaussian * 3) * 3), ("size_mix_weights", f32 * 3), ("size_mix_gain", f32),
    ("sublayer_count", size_t), ("micro_structure", f32 * 2), ("clump_temporal_mix", f32),
    ("size_mix_scale", f32), ("amplitude", f32), ("chroma_mix", f32), ("chroma_shared_weight", f32),
    ("chroma_independent_weight", f32), ("particle_density_min_cmy", f32 * 3), ("uniformity_cmy", f32 * 3),
    ("layer_axis_block_prefix_max", (f32 * 16) * 3), ("recipe_hash", u64), ("density_layers_hash", u64),
    ("hash", u64)])
_dust_names = """cell_width_mm cell_height_mm slot_probability softness_min_mm softness_max_mm
softness_size_cap_fraction support_x_mm support_y_mm fiber_fraction fiber_drift_fraction fiber_first_knot_min
fiber_first_knot_max fiber_second_knot_min fiber_second_knot_max fiber_interior_width_min_fraction
fiber_interior_width_max_fraction diameter_min_mm diameter_bulk_max_mm diameter_max_mm diameter_tail_fraction
fiber_length_min_mm fiber_length_max_mm fiber_width_min_mm fiber_width_max_mm opacity_faint_cumulative
opacity_intermediate_cumulative compact_opacity_min compact_opacity_faint_end compact_opacity_intermediate_end
compact_opacity_max fiber_opacity_min fiber_opacity_faint_end fiber_opacity_intermediate_end fiber_opacity_max
compact_dominant_aspect_min compact_dominant_aspect_max compact_subsidiary_scale_min compact_subsidiary_scale_max
compact_subsidiary_aspect_min compact_subsidiary_aspect_max compact_subsidiary_offset_max
compact_subsidiary_angle_max_radians""".split()
FjDust = _s("FjDust", [(n, f32) for n in _dust_names])
_scratch_names = """cell_width_mm cell_height_mm slot_probability softness_min_mm softness_max_mm
softness_size_cap_fraction support_x_mm support_y_mm length_min_mm length_bulk_max_mm length_max_mm
length_tail_fraction width_min_mm width_bulk_max_mm width_max_mm width_tail_fraction drift_fraction
first_knot_min first_knot_max second_knot_min second_knot_max interior_width_min_fraction
interior_width_max_fraction interior_depth_min_fraction interior_depth_max_fraction endpoint_abrupt_probability
interruption_probability gap_center_min gap_center_max gap_span_min gap_span_max scuff_probability
scuff_length_max_mm scuff_angle_max_radians strength_min strength_max""".split()
FjScratch = _s("FjScratch", [(n, f32) for n in _scratch_names])
FjDefectOrigin = _s("FjDefectOrigin", [("cell_x", i64), ("cell_y", i64), ("local_x_mm", f32),
                                       ("local_y_mm", f32)])
FjFilmEffects = _s("FjFilmEffects", [
    ("render_extent", FjExtent), ("full_frame_extent", FjExtent), ("film_dust", FjDust),
    ("film_scratch", FjScratch), ("gate_dust", FjDust), ("gate_scratch", FjScratch),
    ("origins", FjDefectOrigin * 4), ("sample_step_x_mm", f32), ("sample_step_y_mm", f32),
    ("roi_offset_x", i32), ("roi_offset_y", i32), ("gate_width", i32), ("gate_height", i32),
    ("session_seed", u64), ("clip_token", u64), ("flags", u32), ("weave_dx_px", f32), ("weave_dy_px", f32),
    ("weave_cos_rot", f32), ("weave_sin_rot", f32), ("recipe_hash", u64), ("hash", u64)])
FjStaticNoise = _s("FjStaticNoise", [
    ("stbn", FjByteSpan), ("stbn_width", i32), ("stbn_height", i32), ("stbn_frames", i32),
    ("wang_tiles", FjByteSpan), ("wang_lut", FjByteSpan), ("wang_width", i32), ("wang_height", i32),
    ("wang_tile_count", size_t), ("wang_colors", i32)])
FjPreparedHostData = _s("FjPreparedHostData", [
    ("route", u32), ("capture_polarity", u32), ("film_profile_key", FjStringView),
    ("print_profile_key", FjStringView), ("film_profile_asset_version", u64),
    ("print_profile_asset_version", u64), ("recipe_hash", u64), ("film_exposure", FjFilmExposure),
    ("auto_exposure", FjAutoExposure), ("film_development", FjFilmDevelopment), ("dir_couplers", FjDirCouplers),
    ("scanner_bounds", FjDensityBounds), ("enlarger_film_bounds", FjDensityBounds),
    ("scanner_spectra", FjScannerSpectra), ("scanner_lut", FjScannerLut),
    ("scanner_correction", FjScannerCorrection), ("scanner_post", FjScannerPostEffects),
    ("output_color", FjOutputColor), ("print", FjPrint), ("optics", FjOptics), ("spatial_dir", FjSpatialDir),
    ("grain", FjVisualGrain), ("effects", FjFilmEffects), ("noise", FjStaticNoise)])
FjDiffusionComponents = _s("FjDiffusionComponents", [("lambda_px", f64 * 9), ("red_weights", f64 * 9),
                                                     ("green_weights", f64 * 9), ("blue_weights", f64 * 9)])
FjbTcLutInput = _s("FjbTcLutInput", [("spectra", C.c_void_p), ("sensitivity_rgb", C.POINTER(C.c_float)),
                                     ("reference_illuminant", C.POINTER(C.c_float)), ("projection_white_xyz", f32 * 3),
                                     ("spectral_blur", f32), ("method", u32), ("apply_surface", u32),
                                     ("input_compression", u32), ("surface_rgb", C.POINTER(C.c_float)),
                                     ("hull_xy", C.POINTER(C.c_float)), ("hull_center", f32 * 2),
                                     ("hull_available", u32)])
FJB_STAGE_NAMES = ["auto_exposure", "camera_exposure", "camera_diffusion", "scatter_halation", "spatial_dir",
                   "capture_density", "grain", "print_scan_output", "monolithic", "film_defects",
                   "enlarger_diffusion"]
FjbStageTimes = _s("FjbStageTimes", [("total_ms", f64 * 11), ("frames", u64 * 11)])
FjbScannerLutInput = _s("FjbScannerLutInput", [
    ("eps_c", FjFloatSpan), ("eps_m", FjFloatSpan), ("eps_y", FjFloatSpan), ("weighted_x", FjFloatSpan),
    ("weighted_y", FjFloatSpan), ("weighted_z", FjFloatSpan), ("baseline_min", FjFloatSpan),
    ("range_min_cmy", f32 * 3), ("inverse_span_cmy", f32 * 3), ("sample_count", i32), ("inv_yn", f32),
    ("has_baseline", u32), ("medium", u32), ("resolution", u32)])

# Every record of the public headers, for the layout test.
# print forms of the 81-wavelength contraction (fjb_recipe_set_print_form)
FJB_PRINT_FP32, FJB_PRINT_TENSOR, FJB_PRINT_TENSOR_SPLIT = 0, 1, 2

FJB_DIFFUSION_DIRECT = 0
FJB_DIFFUSION_FFT = 1

FjbFitParams = _s("FjbFitParams", [("exposure_ev", f32 * 3), ("film_gamma", f32 * 3), ("print_gamma", f32 * 3),
                                   ("donor_k", f32 * 3), ("print_ev", f32)])
FJB_FIT_PARAM_NAMES = ["exposure_ev_b", "exposure_ev_g", "exposure_ev_r", "film_gamma_b", "film_gamma_g",
                       "film_gamma_r", "print_gamma_c", "print_gamma_m", "print_gamma_y", "donor_k_b", "donor_k_g",
                       "donor_k_r", "print_ev"]

ALL_RECORDS = [
    FjStatus, FjRenderOutcome, FjErrorBuffer, FjStringView, FjFloatSpan, FjByteSpan, FjCudaContext, FjRect,
    FjExtent, FjImage, FjEffectsGeometry, FjFrame, FjSubmission, FjAbortCallback, FjAutoExposure,
    FjFilmExposure, FjFilmDevelopment, FjDirCouplers, FjDensityBounds, FjScannerSpectra, FjScannerLut,
    FjScannerCorrection, FjScannerPostEffects, FjOutputEncoding, FjOutputColor, FjPrint, FjDiffusion,
    FjHalationGaussian, FjHalationChannel, FjScatterHalation, FjHighlightBoost, FjOptics, FjDirGaussian,
    FjSpatialDir, FjGrainGaussian, FjVisualGrain, FjDust, FjScratch, FjDefectOrigin, FjFilmEffects,
    FjStaticNoise, FjPreparedHostData, FjbScannerLutInput, FjDiffusionComponents, FjbStageTimes, FjbFitParams,
]


class ErrorText:
    """Owns an FjErrorBuffer and its storage."""

    def __init__(self, capacity: int = 1024):
        self._store = C.create_string_buffer(capacity)
        self.buf = FjErrorBuffer(C.cast(self._store, C.c_char_p), capacity, 0)

    @property
    def text(self) -> str:
        return self._store.value.decode("utf-8", "replace")


def float_span(array) -> FjFloatSpan:
    """Span over a contiguous float32 numpy array (the caller keeps it alive)."""
    import numpy as np

    if array is None:
        return FjFloatSpan(None, 0)
    a = np.ascontiguousarray(array, dtype=np.float32)
    if a is not array:
        raise ValueError("float_span needs a contiguous float32 array that outlives the span")
    return FjFloatSpan(a.ctypes.data_as(C.POINTER(f32)), a.size)


def set_floats(field, values) -> None:
    for i, v in enumerate(values):
        field[i] = float(v)
