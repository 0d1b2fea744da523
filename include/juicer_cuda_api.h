/* juicer_cuda_api.h -- the render C-ABI that libjuicer_b200.so exports.
 *
 * This header restates, in this project's own words, the record layouts and the
 * seven entry points of Film-Juicer's native render boundary
 * (native/juicer_cuda_api.h:17-830 in the reference). Field names, types and order
 * are kept identical on purpose: the Rust host fills these records and binds the
 * symbols through rust/film-juicer-plugin/src/cuda/sys.rs:1712-1749, so any change
 * of layout would break the drop-in. tests/test_abi_layout.py pins sizeof/offsetof
 * of every record against an independent ctypes description.
 *
 * Conventions (unchanged from the reference contract):
 *  - every record is a non-owning value; spans borrow caller memory until the call
 *    returns, so the library copies whatever it still needs before returning;
 *  - an empty span is (NULL, 0); counts are element counts;
 *  - image addresses are device addresses; rows are row_bytes apart.
 */
#ifndef JUICER_CUDA_API_H
#define JUICER_CUDA_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct FjCuda FjCuda; /* opaque owner returned by fj_cuda_create */

/* Status categories (reference native/juicer_cuda_api.h:19-27). */
#define FJ_STATUS_SUCCESS 0U
#define FJ_STATUS_CANCELLED 1U
#define FJ_STATUS_UNSUPPORTED_INPUT 2U
#define FJ_STATUS_PREPARATION_FAILURE 3U
#define FJ_STATUS_ALLOCATION_FAILURE 4U
#define FJ_STATUS_CUDA_FAILURE 5U
#define FJ_STATUS_CUFFT_FAILURE 6U
#define FJ_STATUS_CONTEXT_LOSS 7U
#define FJ_STATUS_INTERNAL_FAILURE 8U
/* Which API produced native_code (reference :28-31). */
#define FJ_API_NONE 0U
#define FJ_API_CUDA_RUNTIME 1U
#define FJ_API_CUDA_DRIVER 2U
#define FJ_API_CUFFT 3U

typedef struct FjStatus {
    uint32_t category;
    uint32_t api;
    int32_t native_code;
} FjStatus;

/* Render flag: a DIR receiver evaluation failed on the device during this frame. */
#define FJ_RENDER_DEFERRED_DIR_ERROR 1U
typedef struct FjRenderOutcome {
    FjStatus status;
    uint32_t flags;
} FjRenderOutcome;

/* Caller-owned diagnostic text. capacity counts the trailing NUL that is always
 * written when capacity > 0; length excludes it. Truncation never alters status. */
typedef struct FjErrorBuffer {
    char* data;
    size_t capacity;
    size_t length;
} FjErrorBuffer;

typedef struct FjStringView {
    const char* data;
    size_t count;
} FjStringView;

#define FJ_PATH_UNIX_BYTES 1U
#define FJ_PATH_WINDOWS_WIDE 2U
typedef struct FjPathView {
    const void* data;
    size_t count;
    uint32_t encoding;
} FjPathView;

typedef struct FjFloatSpan {
    const float* data;
    size_t count;
} FjFloatSpan;

typedef struct FjByteSpan {
    const uint8_t* data;
    size_t count;
} FjByteSpan;

typedef struct FjCudaContext {
    int32_t device_id;
    uintptr_t context;
} FjCudaContext;

typedef struct FjRect {
    int32_t x1;
    int32_t y1;
    int32_t x2; /* exclusive */
    int32_t y2; /* exclusive */
} FjRect;

typedef struct FjExtent {
    int32_t x;
    int32_t y;
    int32_t width;
    int32_t height;
} FjExtent;

#define FJ_COMPONENTS_UNKNOWN 0U
#define FJ_COMPONENTS_RGB 3U
#define FJ_COMPONENTS_RGBA 4U
#define FJ_DEPTH_UNKNOWN 0U
#define FJ_DEPTH_FLOAT32 1U
#define FJ_FRAME_STREAM_PRESENT 1U
#define FJ_FRAME_TRACE_INFO 2U
#define FJ_FRAME_TRACE_VERBOSE 4U

typedef struct FjImage {
    uintptr_t address; /* device pointer of pixel (bounds.x1, bounds.y1) */
    FjRect bounds;
    ptrdiff_t row_bytes;
    uint32_t components; /* FJ_COMPONENTS_* */
    uint32_t depth;      /* FJ_DEPTH_* */
} FjImage;

typedef struct FjEffectsGeometry {
    FjExtent pixel_definition;
    double canonical_x;
    double canonical_y;
    double canonical_width;
    double canonical_height;
    double scale_x;
    double scale_y;
    double pixel_aspect_ratio;
} FjEffectsGeometry;

typedef struct FjFrame {
    FjImage source;
    FjImage destination;
    FjRect render_window;
    FjRect full_frame_extent;
    uintptr_t stream; /* cudaStream_t when FJ_FRAME_STREAM_PRESENT */
    uint32_t flags;   /* FJ_FRAME_* */
    float pixel_size_um;
    double time_frames;
    double frame_rate;
    uint64_t session_seed;
    uint64_t clip_token;
    FjEffectsGeometry effects_geometry;
} FjFrame;

typedef struct FjSubmission {
    uint64_t instance_token;
    uint64_t frame_token;
    uint64_t submission_id;
    uint64_t upload_core_hash;
    uint64_t dir_hash;
    uint64_t scanner_hash;
    uint64_t auto_exposure_hash;
} FjSubmission;

#define FJ_ABORT_CONTINUE 0U
#define FJ_ABORT_REQUESTED 1U
typedef uint32_t (*FjAbortQuery)(void* user);
typedef struct FjAbortCallback {
    FjAbortQuery query; /* may be NULL: never abort */
    void* user;
} FjAbortCallback;

#define FJ_ROUTE_NEGATIVE_DIRECT 0U
#define FJ_ROUTE_NEGATIVE_PRINT 1U
#define FJ_ROUTE_POSITIVE_DIRECT 2U
#define FJ_ROUTE_POSITIVE_PRINT 3U
#define FJ_POLARITY_NEGATIVE 0U
#define FJ_POLARITY_POSITIVE 1U
#define FJ_POLARITY_UNSUPPORTED 2U
#define FJ_RAW_HANATOS_2025 0U
#define FJ_RAW_MALLETT_2019 1U
#define FJ_RAW_ARCTIC_2026_BETA04 2U
#define FJ_INPUT_DWG 0U
#define FJ_INPUT_BT2020 1U
#define FJ_INPUT_ACES2065_1 2U
#define FJ_INPUT_SRGB_REC709 3U
#define FJ_FILM_DECODE_CCTF 1U
#define FJ_FILM_ADAPT_INPUT 2U
#define FJ_FILM_AUTO_EXPOSURE 4U
#define FJ_METER_CENTER_WEIGHTED 0U
#define FJ_METER_AVERAGE 1U
#define FJ_METER_MEDIAN 2U
#define FJ_METER_PARTIAL 3U
#define FJ_METER_MATRIX 4U
#define FJ_METER_MULTI_ZONE 5U
#define FJ_METER_HIGHLIGHT_WEIGHTED 6U

typedef struct FjAutoExposure {
    FjRect source_bounds;
    FjRect meter_bounds;
    int32_t preview_width;
    int32_t preview_height;
    uint32_t method; /* FJ_METER_* */
    uint64_t hash;
} FjAutoExposure;

typedef struct FjFilmExposure {
    uint32_t input_color_space; /* FJ_INPUT_* */
    uint32_t method;            /* FJ_RAW_* */
    uint32_t flags;             /* FJ_FILM_* */
    float manual_exposure_ev;
    float route_correction_scale;
    float mallett_green_midgray_scale;
    float input_rgb_to_xyz[9];
    float input_xyz_adapt[9];
    float xyz_to_linear_srgb[9];
    FjFloatSpan sensitivity_rgb;    /* float[81*3], wavelength-major R,G,B */
    FjFloatSpan tc_lut_rgba;        /* float[192*192*4], [c][m][R,G,B,pad] */
    FjFloatSpan mallett_illuminant; /* float[81] */
    FjFloatSpan mallett_basis;      /* float[81*3] */
    uint64_t sensitivity_hash;
    uint64_t tc_lut_hash;
    uint64_t hash;
} FjFilmExposure;

typedef struct FjFilmDevelopment {
    FjFloatSpan log_exposure;            /* float[N], ascending log10 exposure */
    FjFloatSpan density_rgb;             /* float[N*3], [sample][R,G,B] */
    FjFloatSpan density_layers[3][3];    /* per layer/channel float[N] (grain) */
    float gamma_rgb[3];
    uint64_t density_curves_hash;
    uint64_t density_layers_hash;
    uint64_t hash;
} FjFilmDevelopment;

#define FJ_DIR_INACTIVE 0U
#define FJ_DIR_NEGATIVE_DONOR_LANGMUIR 1U
#define FJ_DIR_POSITIVE_RECEIVER_LANGMUIR 2U
typedef struct FjDirCouplers {
    uint32_t mode;
    float matrix_rgb[9]; /* [donor R,G,B][receiver R,G,B] */
    float density_max_rgb[3];
    float density_ref_rgb[3];
    float donor_k_rgb[3];
    float receiver_c_ref_rgb[3];
    float receiver_kr_rgb[3];
    FjFloatSpan compensated_axes_rgb[3]; /* three float[N] log10 exposure axes */
    uint64_t compensated_axes_hash;
    uint64_t hash;
} FjDirCouplers;

typedef struct FjDensityBounds {
    float min_cmy[3];
    float inv_span_cmy[3];
    uint64_t hash;
} FjDensityBounds;

typedef struct FjScannerSpectra {
    FjFloatSpan dye_y; /* float[81] each */
    FjFloatSpan dye_m;
    FjFloatSpan dye_c;
    FjFloatSpan weighted_x;
    FjFloatSpan weighted_y;
    FjFloatSpan weighted_z;
    FjFloatSpan base_density; /* float[81] or empty */
    float inverse_y_normalization;
} FjScannerSpectra;

typedef struct FjScannerLut {
    uint64_t density_bounds_hash;
    uint32_t resolution;
    uint64_t hash;
} FjScannerLut;

#define FJ_CORRECTION_ACTIVE 1U
typedef struct FjScannerCorrection {
    uint32_t flags;
    float xyz_slope;
    float xyz_offset;
    float exposure_scale;
} FjScannerCorrection;

#define FJ_POST_GLARE 1U
typedef struct FjScannerPostEffects {
    uint32_t flags;
    float glare_percent;
    float glare_roughness;
    float glare_blur_sigma_px;
    int32_t glare_blur_radius;
    float lens_blur_sigma_px;
    int32_t lens_blur_radius;
    float unsharp_sigma_px;
    int32_t unsharp_radius;
    float unsharp_amount;
    uint64_t hash;
} FjScannerPostEffects;

#define FJ_OUTPUT_SRGB 0U
#define FJ_OUTPUT_DCI_P3 1U
#define FJ_OUTPUT_DISPLAY_P3 2U
#define FJ_OUTPUT_ADOBE_RGB 3U
#define FJ_OUTPUT_BT2020 4U
#define FJ_OUTPUT_PROPHOTO_RGB 5U
#define FJ_OUTPUT_ACES2065_1 6U
#define FJ_OUTPUT_DWG_INTERMEDIATE 7U
#define FJ_OUTPUT_REC709 8U
#define FJ_COLOR_ENCODE_CCTF 1U
#define FJ_COLOR_INPUT_IS_OUTPUT_SPACE 2U
#define FJ_COLOR_GAMUT_COMPRESSION 4U
#define FJ_OUTPUT_ENCODING_SCHEMA 1U
#define FJ_CCTF_LINEAR 0U
#define FJ_CCTF_GAMMA 1U
#define FJ_CCTF_SRGB 2U
#define FJ_CCTF_BT2020 3U
#define FJ_CCTF_PROPHOTO 4U
#define FJ_CCTF_DWG_INTERMEDIATE 5U
typedef struct FjOutputEncoding {
    uint32_t schema;
    uint32_t cctf_kind;
    float gamma;
    float a;
    float b;
    float c;
    float d;
    float linear_cutoff;
    float dwg_to_output[9];
} FjOutputEncoding;

typedef struct FjOutputColor {
    float cat02[9];
    float xyz_to_rgb[9];
    float illuminant_xyz[3];
    uint32_t color_space; /* FJ_OUTPUT_* */
    uint32_t flags;       /* FJ_COLOR_* */
    float native_rgb_to_d65_xyz[9];
    float d65_xyz_to_native_rgb[9];
    float lightness_knee[3]; /* threshold, limit, power */
    float chroma_knee[3];
    FjFloatSpan gamut_cmax; /* float[64*720], [lightness][hue] max OkLab chroma */
    uint64_t gamut_table_hash;
    uint64_t gamut_recipe_hash;
    FjOutputEncoding encoding;
} FjOutputColor;

#define FJ_PRINT_PREFLASH 1U
typedef struct FjPrint {
    FjFloatSpan film_density_cmy;  /* float[81*3], [wavelength][C,M,Y] */
    FjFloatSpan film_base_density; /* float[81] */
    FjFloatSpan sensitivity_cmy;   /* float[81*3] */
    FjFloatSpan log_exposure;      /* float[N] */
    FjFloatSpan density_cmy;       /* float[N*3] */
    FjFloatSpan main_illuminant;   /* float[81] */
    FjFloatSpan preflash_illuminant;
    uint32_t flags;
    float main_cc_cmy[3];
    float preflash_cc_cmy[3];
    float exposure;
    float preflash_exposure;
    float preflash_raw_cmy[3];
    float normalizer;
    uint64_t film_density_hash;
    uint64_t profile_tables_hash;
    uint64_t main_illuminant_hash;
    uint64_t preflash_illuminant_hash;
    uint64_t preflash_raw_hash;
    uint64_t balance_hash;
    uint64_t hash;
} FjPrint;

#define FJ_DIFFUSION_GLIMMERGLASS 0U
#define FJ_DIFFUSION_BLACK_PRO_MIST 1U
#define FJ_DIFFUSION_PRO_MIST 2U
#define FJ_DIFFUSION_CINEBLOOM 3U
#define FJ_OPTICS_CAMERA_DIFFUSION 1U
#define FJ_OPTICS_ENLARGER_DIFFUSION 2U
#define FJ_OPTICS_SCATTER_HALATION 4U
#define FJ_OPTICS_HIGHLIGHT_BOOST 8U

typedef struct FjDiffusion {
    uint32_t family;
    double scatter_fraction;
    double group_weights[3];
    double group_lambda_um[3];
    double warmth;
    double spatial_scale;
    double pixel_size_um;
    int32_t radius_px;
    uint64_t sample_hash;
    uint64_t hash;
} FjDiffusion;

#define FJ_HALATION_IDENTITY 0U
#define FJ_HALATION_FIR_REFLECT 1U
#define FJ_HALATION_YVV_REPLICATE 2U
#define FJ_HALATION_YVV_REPLICATE_FACTORED 3U
#define FJ_HALATION_TAIL_COMPONENTS 3U
#define FJ_HALATION_MAX_BOUNCES 5U
typedef struct FjHalationGaussian {
    uint32_t kind;
    int32_t radius;
    float fir_weights[19];
    float yvv[4]; /* legacy: B,B1,B2,B3; factored: h,g,t,0 */
} FjHalationGaussian;

typedef struct FjHalationChannel {
    FjHalationGaussian core;
    FjHalationGaussian tail[FJ_HALATION_TAIL_COMPONENTS];
    FjHalationGaussian bounce[FJ_HALATION_MAX_BOUNCES];
    float total_strength;
    float tail_weight;
} FjHalationChannel;

typedef struct FjScatterHalation {
    uint64_t recipe_hash;
    float scatter_amount;
    uint32_t bounce_count;
    float bounce_weights[FJ_HALATION_MAX_BOUNCES];
    uint32_t renormalize;
    FjHalationChannel channels[3]; /* R,G,B */
} FjScatterHalation;

typedef struct FjHighlightBoost {
    uint64_t recipe_hash;
    double protection;
    double sharpness;
    double peak_gain;
} FjHighlightBoost;

typedef struct FjOptics {
    uint32_t flags; /* FJ_OPTICS_* */
    FjExtent full_frame;
    FjDiffusion camera;
    FjDiffusion enlarger;
    uint64_t diffusion_hash;
    FjScatterHalation scatter_halation;
    FjHighlightBoost highlight_boost;
} FjOptics;

#define FJ_DIR_OPERATOR_NONE 0U
#define FJ_DIR_OPERATOR_IDENTITY 1U
#define FJ_DIR_OPERATOR_FIR_REFLECT 2U
#define FJ_DIR_OPERATOR_YVV_REFLECT 3U
typedef struct FjDirGaussian {
    float sigma_px;
    float weight;
    int32_t radius;
    uint32_t reference_operator; /* FJ_DIR_OPERATOR_* */
    double feedforward;
    double feedback[3];
    double normalization_denominator;
    double feedforward_numerator;
    double feedback_numerators[3];
    double boundary_truncation_accuracy;
    double boundary_certification_tolerance;
    uint32_t boundary_derivation_version;
} FjDirGaussian;

typedef struct FjSpatialDir {
    FjExtent render_extent;
    FjExtent full_frame_extent;
    FjExtent filter_domain_extent;
    size_t component_count; /* 0..4 */
    FjDirGaussian components[4];
    uint64_t recipe_hash;
    uint64_t hash;
} FjSpatialDir;

#define FJ_GRAIN_ACTIVE 1U
#define FJ_GRAIN_SUBLAYERS 2U
#define FJ_GRAIN_FULL_FRAME 4U
#define FJ_GRAIN_AXIS_FINITE_C 8U
#define FJ_GRAIN_AXIS_FINITE_M 16U
#define FJ_GRAIN_AXIS_FINITE_Y 32U
#define FJ_GRAIN_DEBUG_OFF 0U
#define FJ_GRAIN_DEBUG_DELTA_MIX 1U
#define FJ_GRAIN_DEBUG_DELTA_FINE 2U
#define FJ_GRAIN_DEBUG_DELTA_COARSE 3U
#define FJ_GRAIN_DEBUG_DELTA_FINE_RAW 4U
#define FJ_GRAIN_DEBUG_DELTA_COARSE_RAW 5U
#define FJ_GRAIN_DEBUG_MEAN_DENSITY 6U

typedef struct FjGrainGaussian {
    float sigma_px;
    int32_t radius;
    uint64_t hash;
} FjGrainGaussian;

typedef struct FjVisualGrain {
    uint32_t flags;
    uint32_t debug_view;
    FjExtent render_extent;
    FjExtent full_frame_extent;
    float pixel_size_um;
    int64_t frame0;
    float frame_alpha;
    uint64_t seed_base;
    uint64_t seed_base_next;
    uint64_t session_seed;
    uint64_t clip_token;
    int32_t pitch_px;
    int32_t breathing_period_frames;
    int32_t clump_morph_period_frames;
    float wang_cell_mm;
    float breathing_amplitude;
    float breathing_cell_um_small;
    float breathing_cell_um_large;
    float breathing_mix;
    float breathing_drift_um_per_frame;
    float debug_scale;
    float density_max_cmy[3];
    float n_particles_cmy[3];
    float od_particle_cmy[3];
    float density_min_layers[3][3];
    float density_max_layers[3][3];
    float n_particles_layers[3][3];
    float od_particle_layers[3][3];
    FjGrainGaussian correlation[3];
    FjGrainGaussian dye_cloud[3][3];
    float size_mix_weights[3];
    float size_mix_gain;
    size_t sublayer_count;
    float micro_structure[2];
    float clump_temporal_mix;
    float size_mix_scale;
    float amplitude;
    float chroma_mix;
    float chroma_shared_weight;
    float chroma_independent_weight;
    float particle_density_min_cmy[3];
    float uniformity_cmy[3];
    float layer_axis_block_prefix_max[3][16];
    uint64_t recipe_hash;
    uint64_t density_layers_hash;
    uint64_t hash;
} FjVisualGrain;

typedef struct FjDust {
    float cell_width_mm;
    float cell_height_mm;
    float slot_probability;
    float softness_min_mm;
    float softness_max_mm;
    float softness_size_cap_fraction;
    float support_x_mm;
    float support_y_mm;
    float fiber_fraction;
    float fiber_drift_fraction;
    float fiber_first_knot_min;
    float fiber_first_knot_max;
    float fiber_second_knot_min;
    float fiber_second_knot_max;
    float fiber_interior_width_min_fraction;
    float fiber_interior_width_max_fraction;
    float diameter_min_mm;
    float diameter_bulk_max_mm;
    float diameter_max_mm;
    float diameter_tail_fraction;
    float fiber_length_min_mm;
    float fiber_length_max_mm;
    float fiber_width_min_mm;
    float fiber_width_max_mm;
    float opacity_faint_cumulative;
    float opacity_intermediate_cumulative;
    float compact_opacity_min;
    float compact_opacity_faint_end;
    float compact_opacity_intermediate_end;
    float compact_opacity_max;
    float fiber_opacity_min;
    float fiber_opacity_faint_end;
    float fiber_opacity_intermediate_end;
    float fiber_opacity_max;
    float compact_dominant_aspect_min;
    float compact_dominant_aspect_max;
    float compact_subsidiary_scale_min;
    float compact_subsidiary_scale_max;
    float compact_subsidiary_aspect_min;
    float compact_subsidiary_aspect_max;
    float compact_subsidiary_offset_max;
    float compact_subsidiary_angle_max_radians;
} FjDust;

typedef struct FjScratch {
    float cell_width_mm;
    float cell_height_mm;
    float slot_probability;
    float softness_min_mm;
    float softness_max_mm;
    float softness_size_cap_fraction;
    float support_x_mm;
    float support_y_mm;
    float length_min_mm;
    float length_bulk_max_mm;
    float length_max_mm;
    float length_tail_fraction;
    float width_min_mm;
    float width_bulk_max_mm;
    float width_max_mm;
    float width_tail_fraction;
    float drift_fraction;
    float first_knot_min;
    float first_knot_max;
    float second_knot_min;
    float second_knot_max;
    float interior_width_min_fraction;
    float interior_width_max_fraction;
    float interior_depth_min_fraction;
    float interior_depth_max_fraction;
    float endpoint_abrupt_probability;
    float interruption_probability;
    float gap_center_min;
    float gap_center_max;
    float gap_span_min;
    float gap_span_max;
    float scuff_probability;
    float scuff_length_max_mm;
    float scuff_angle_max_radians;
    float strength_min;
    float strength_max;
} FjScratch;

typedef struct FjDefectOrigin {
    int64_t cell_x;
    int64_t cell_y;
    float local_x_mm;
    float local_y_mm;
} FjDefectOrigin;

#define FJ_EFFECTS_WEAVE 1U
#define FJ_EFFECTS_FILM 2U
#define FJ_EFFECTS_GATE_TRANSMITTANCE 4U
#define FJ_EFFECTS_GATE_OUTPUT 8U
#define FJ_EFFECTS_FULL_FRAME 16U
typedef struct FjFilmEffects {
    FjExtent render_extent;
    FjExtent full_frame_extent;
    FjDust film_dust;
    FjScratch film_scratch;
    FjDust gate_dust;
    FjScratch gate_scratch;
    FjDefectOrigin origins[4];
    float sample_step_x_mm;
    float sample_step_y_mm;
    int32_t roi_offset_x;
    int32_t roi_offset_y;
    int32_t gate_width;
    int32_t gate_height;
    uint64_t session_seed;
    uint64_t clip_token;
    uint32_t flags;
    float weave_dx_px;
    float weave_dy_px;
    float weave_cos_rot;
    float weave_sin_rot;
    uint64_t recipe_hash;
    uint64_t hash;
} FjFilmEffects;

typedef struct FjStaticNoise {
    FjByteSpan stbn; /* uint8_t[frames][height][width] */
    int32_t stbn_width;
    int32_t stbn_height;
    int32_t stbn_frames;
    FjByteSpan wang_tiles; /* uint8_t[tile][height][width] */
    FjByteSpan wang_lut;   /* uint8_t[colors^4] */
    int32_t wang_width;
    int32_t wang_height;
    size_t wang_tile_count;
    int32_t wang_colors;
} FjStaticNoise;

/* Everything the host prepared for one render call. */
typedef struct FjPreparedHostData {
    uint32_t route;            /* FJ_ROUTE_* */
    uint32_t capture_polarity; /* FJ_POLARITY_* */
    FjStringView film_profile_key;
    FjStringView print_profile_key;
    uint64_t film_profile_asset_version;
    uint64_t print_profile_asset_version;
    uint64_t recipe_hash;
    FjFilmExposure film_exposure;
    FjAutoExposure auto_exposure;
    FjFilmDevelopment film_development;
    FjDirCouplers dir_couplers;
    FjDensityBounds scanner_bounds;
    FjDensityBounds enlarger_film_bounds;
    FjScannerSpectra scanner_spectra;
    FjScannerLut scanner_lut;
    FjScannerCorrection scanner_correction;
    FjScannerPostEffects scanner_post;
    FjOutputColor output_color;
    FjPrint print;
    FjOptics optics;
    FjSpatialDir spatial_dir;
    FjVisualGrain grain;
    FjFilmEffects effects;
    FjStaticNoise noise;
} FjPreparedHostData;

/* Creates the single library owner (reference native/juicer_cuda_api.h:794). */
FjStatus fj_cuda_create(FjCuda** out_cuda, FjErrorBuffer* error);
/* Cheap liveness check of the owner (reference :797). */
FjStatus fj_cuda_check_terminal(FjCuda* cuda, FjErrorBuffer* error);
/* Validates the frame and reports the device/context it lives on (reference :802). */
FjStatus fj_cuda_inspect(FjCuda* cuda, const FjFrame* frame, FjCudaContext* out_context, FjErrorBuffer* error);
/* Renders one frame on frame->stream (reference :809). */
FjRenderOutcome fj_cuda_render(FjCuda* cuda, const FjCudaContext* context, const FjFrame* frame,
                               const FjSubmission* submission, const FjPreparedHostData* prepared,
                               FjAbortCallback abort_callback, FjErrorBuffer* error);
/* Drops per-instance cached state (reference :812). */
FjStatus fj_cuda_retire_instance(FjCuda* cuda, uint64_t instance_token, FjErrorBuffer* error);
/* Releases device resources; the handle stays valid for fj_cuda_destroy (reference :818). */
FjStatus fj_cuda_shutdown(FjCuda* cuda, FjErrorBuffer* error);
/* Consumes the handle (reference :830). */
FjStatus fj_cuda_destroy(FjCuda* cuda, FjErrorBuffer* error);

#ifdef __cplusplus
}
#endif

#endif /* JUICER_CUDA_API_H */
