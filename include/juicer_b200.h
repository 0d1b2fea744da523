/* juicer_b200.h -- stage-level entry points of libjuicer_b200.so.
 *
 * fj_cuda_render (juicer_cuda_api.h) renders a whole frame. The functions below
 * expose the same device work one stage at a time, for hosts that schedule stages
 * themselves and for parity testing. Every image/plane pointer is a device address;
 * every function enqueues on `stream` (a cudaStream_t, 0 = legacy default stream)
 * and returns without synchronising unless it says otherwise. No torch or CUDA C++
 * types appear in these signatures.
 */
#ifndef JUICER_B200_H
#define JUICER_B200_H

#include <stddef.h>
#include <stdint.h>

#include "juicer_cuda_api.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Device-resident tables of one prepared recipe (TC LUT, curves, print spectra,
 * scanner PCHIP LUT, gamut boundary). Opaque. */
typedef struct FjbRecipe FjbRecipe;

/* Uploads the tables named by `prepared` and builds the scanner LUT on the device
 * (FP64). Replaces the reference's per-recipe preparation
 * (src/Cuda/JuicerCudaExecutor.cpp:2873 Root::prepare_cuda_frame with the
 * scanner-LUT host callback native/juicer_host_preparation.cpp:28). Synchronises
 * `stream` before returning so that the borrowed spans may be released. */
FjStatus fjb_recipe_create(const FjPreparedHostData* prepared, void* stream, FjbRecipe** out_recipe,
                           FjErrorBuffer* error);
FjStatus fjb_recipe_destroy(FjbRecipe* recipe, FjErrorBuffer* error);

/* Device scalar read by the exposure step as the auto-exposure scale (NULL = 1). */
FjStatus fjb_recipe_set_exposure_scale_device(FjbRecipe* recipe, const float* device_scale, FjErrorBuffer* error);

/* Arithmetic of the print exposure's 81-wavelength contraction for this recipe's
 * print stages from density planes (fjb_render_from_density*, fjb_print_raw and the
 * staged schedule of fj_cuda_render): FJB_PRINT_FP32 (default; FP32 FMAs, the
 * reference's arithmetic), FJB_PRINT_TENSOR (tcgen05 BF16 tensor-core tiles with FP32
 * accumulation: densities and spectra as hi + lo BF16 pairs, transmittances as one
 * BF16) or FJB_PRINT_TENSOR_SPLIT (transmittances as hi + lo pairs too). No
 * counterpart in the reference, which has the FP32 form only
 * (src/Cuda/JuicerCudaDeviceHelpers.cuh:866-935). */
#define FJB_PRINT_FP32 0
#define FJB_PRINT_TENSOR 1
#define FJB_PRINT_TENSOR_SPLIT 2
FjStatus fjb_recipe_set_print_form(FjbRecipe* recipe, int32_t form, FjErrorBuffer* error);

/* The print exposure's spectral integral raw_c = sum_l 10^-D(l) I(l) S_c(l) of
 * density planes C, M, Y into planes raw C, M, Y (before dust, normaliser, preflash
 * and exposure), in the recipe's print form: the per-stage precision check of the
 * tensor-core form (reference print_spectral_integrate_device,
 * src/Cuda/JuicerCudaDeviceHelpers.cuh:866). Print route only. */
FjStatus fjb_print_raw(FjbRecipe* recipe, const float* density_c, const float* density_m, const float* density_y,
                       float* raw_c, float* raw_m, float* raw_y, int32_t width, int32_t height, void* stream,
                       FjErrorBuffer* error);

/* Enlarger diffusion, stage by stage (reference
 * src/Cuda/Scan/JuicerCudaScanPipeline.cu:2924 juicer_cuda_print_focused_enlarger_linear_exposure
 * and :2943 juicer_cuda_print_focused_develop_from_enlarger_linear). The print-linear
 * exposure of capture density planes C, M, Y (dust: film dust transmittance plane or
 * NULL) into planes C-, M-, Y-forming (red-, green-, blue-sensitive layers of the
 * paper: the R, G, B planes of fjb_diffusion with the enlarger record); after the
 * diffusion, the print density C, M, Y from those planes (may be the same buffers);
 * then the scan and output encoding of print density planes. Print route only. */
FjStatus fjb_enlarger_linear_exposure(FjbRecipe* recipe, const float* density_c, const float* density_m,
                                      const float* density_y, const float* dust, float* linear_c, float* linear_m,
                                      float* linear_y, int32_t width, int32_t height, void* stream,
                                      FjErrorBuffer* error);
FjStatus fjb_enlarger_develop(FjbRecipe* recipe, const float* linear_c, const float* linear_m, const float* linear_y,
                              float* density_c, float* density_m, float* density_y, int32_t width, int32_t height,
                              void* stream, FjErrorBuffer* error);
FjStatus fjb_render_from_print_density(FjbRecipe* recipe, const float* density_c, const float* density_m,
                                       const float* density_y, const float* src, ptrdiff_t src_row_bytes, float* dst,
                                       ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                       void* stream, FjErrorBuffer* error);

/* Parameter fitting (no counterpart in the reference, which renders only): the
 * per-pixel chain of the recipe (camera exposure, film curves, runtime DIR, print
 * exposure and curves on the print route, scanner LUT, correction and colour
 * matrices) as a function of the parameters below, with its output the scanner's
 * linear output RGB (before output gamut compression and encoding), and the
 * hand-written adjoint of that chain. The default parameters (fjb_fit_defaults)
 * reproduce the recipe. Channel orders: exposure_ev, film_gamma, donor_k B, G, R;
 * print_gamma C, M, Y. */
typedef struct FjbFitParams {
    float exposure_ev[3]; /* film exposure of each layer times 2^ev */
    float film_gamma[3];  /* gamma factor of the film and compensated curves */
    float print_gamma[3]; /* gamma factor of the print curves (1 = the recipe's) */
    float donor_k[3];     /* negative-donor Langmuir knee (> 0) */
    float print_ev;       /* print exposure times 2^ev */
} FjbFitParams;
FjStatus fjb_fit_defaults(FjbRecipe* recipe, FjbFitParams* out, FjErrorBuffer* error);
/* Linear output RGB planes of the source image (NaN where the chain rejects a pixel). */
FjStatus fjb_fit_forward(FjbRecipe* recipe, const FjbFitParams* params, const float* src, ptrdiff_t src_row_bytes,
                         uint32_t components, float* out_r, float* out_g, float* out_b, int32_t width, int32_t height,
                         void* stream, FjErrorBuffer* error);
/* grad_params[13] (device, FP64, FjbFitParams order) = sum over pixels of
 * grad_rgb^T d rgb / d params: the adjoint recomputes each pixel's forward values,
 * the 81 print transmittances included, instead of storing them. `scratch` holds
 * fjb_fit_scratch_bytes() bytes of device memory (per-block partial sums, reduced in
 * a fixed order: the result is deterministic). */
size_t fjb_fit_scratch_bytes(void);
FjStatus fjb_fit_vjp(FjbRecipe* recipe, const FjbFitParams* params, const float* src, ptrdiff_t src_row_bytes,
                     uint32_t components, const float* grad_r, const float* grad_g, const float* grad_b,
                     int32_t width, int32_t height, double* grad_params, void* scratch, size_t scratch_bytes,
                     void* stream, FjErrorBuffer* error);
/* The same chain from carrier planes (film exposure B, G, R before the route
 * correction, as fjb_camera_exposure writes it and the optics stages leave it; row
 * stride in floats) instead of the source RGB: on frames with camera diffusion and
 * scatter/halation, whose stages are linear in the carrier, the exposure parameters
 * scale the carrier after them exactly as before them. fjb_fit_vjp_carrier also
 * writes d <grad_rgb, rgb> / d carrier into grad_carrier_* (all three or none; dense
 * width x height planes), the cotangent for the optics stages' own parameters. */
FjStatus fjb_fit_forward_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                 const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                 float* out_r, float* out_g, float* out_b, int32_t width, int32_t height, void* stream,
                                 FjErrorBuffer* error);
FjStatus fjb_fit_vjp_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                             const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                             const float* grad_r, const float* grad_g, const float* grad_b, int32_t width,
                             int32_t height, double* grad_params, float* grad_carrier_b, float* grad_carrier_g,
                             float* grad_carrier_r, void* scratch, size_t scratch_bytes, void* stream,
                             FjErrorBuffer* error);
/* Spatial DIR (negative-donor couplers), in three steps around the frame's DIR filter
 * (fjb_spatial_dir_blur): fjb_fit_dir_source_carrier writes the donor corrections of
 * the B, G, R receivers (planes Y, M, C) for theta; the caller filters them;
 * fjb_fit_forward_spatial_carrier develops with the filtered corrections. The adjoint
 * runs backwards: fjb_fit_vjp_spatial_carrier gives the theta gradient of the
 * development, the carrier gradient planes and d L / d filtered correction
 * (grad_filtered_*); the filter is symmetric (its own adjoint), so the caller filters
 * that cotangent and fjb_fit_dir_source_vjp_carrier adds the source stage's theta
 * gradient (into its own grad_params) and ADDS its carrier gradient into grad_carrier_*.
 * Every plane uses carrier_stride. */
FjStatus fjb_fit_dir_source_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                    const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                    float* corr_y, float* corr_m, float* corr_c, int32_t width, int32_t height,
                                    void* stream, FjErrorBuffer* error);
FjStatus fjb_fit_forward_spatial_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                         const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                         const float* filtered_y, const float* filtered_m, const float* filtered_c,
                                         float* out_r, float* out_g, float* out_b, int32_t width, int32_t height,
                                         void* stream, FjErrorBuffer* error);
FjStatus fjb_fit_vjp_spatial_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                     const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                     const float* filtered_y, const float* filtered_m, const float* filtered_c,
                                     const float* grad_r, const float* grad_g, const float* grad_b, int32_t width,
                                     int32_t height, double* grad_params, float* grad_carrier_b, float* grad_carrier_g,
                                     float* grad_carrier_r, float* grad_filtered_y, float* grad_filtered_m,
                                     float* grad_filtered_c, void* scratch, size_t scratch_bytes, void* stream,
                                     FjErrorBuffer* error);
FjStatus fjb_fit_dir_source_vjp_carrier(FjbRecipe* recipe, const FjbFitParams* params, const float* carrier_b,
                                        const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                                        const float* grad_corr_y, const float* grad_corr_m, const float* grad_corr_c,
                                        int32_t width, int32_t height, double* grad_params, float* grad_carrier_b,
                                        float* grad_carrier_g, float* grad_carrier_r, void* scratch,
                                        size_t scratch_bytes, void* stream, FjErrorBuffer* error);

/* Device error word (bit 0 scan failure, bit 8 DIR failure, bits 9..11 DIR
 * channels B,G,R, bit 16 a tensor-core wait of the print stage gave up). Cleared by fjb_recipe_clear_flags, read by fjb_recipe_read_flags
 * (which synchronises `stream`). */
FjStatus fjb_recipe_clear_flags(FjbRecipe* recipe, void* stream, FjErrorBuffer* error);
FjStatus fjb_recipe_read_flags(FjbRecipe* recipe, void* stream, uint32_t* out_flags, FjErrorBuffer* error);

/* Fused per-pixel chain, source RGB(A) float32 -> encoded output RGB(A) float32,
 * for the direct and print routes with runtime DIR (reference
 * src/Cuda/Scan/JuicerCudaScanPipeline.cu:2244 juicer_cuda_negative_pipeline and
 * :3759 juicer_cuda_print_pipeline). components is 3 or 4 for both images. */
FjStatus fjb_render_pixels(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, float* dst,
                           ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                           void* stream, FjErrorBuffer* error);

/* Camera exposure to carrier planes B, G, R (stride in floats), without the route
 * correction (reference src/Cuda/Film/JuicerCudaFilmPipeline.cu:3103). */
FjStatus fjb_camera_exposure(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, uint32_t components,
                             int32_t width, int32_t height, float* carrier_b, float* carrier_g, float* carrier_r,
                             ptrdiff_t carrier_stride, void* stream, FjErrorBuffer* error);

/* Carrier planes (may be NULL: then `src` is exposed) -> capture density planes
 * C, M, Y (reference :2880 juicer_cuda_direct_focused_capture_density). */
FjStatus fjb_capture_density(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, uint32_t components,
                             const float* carrier_b, const float* carrier_g, const float* carrier_r,
                             ptrdiff_t carrier_stride, int32_t width, int32_t height, float* density_c,
                             float* density_m, float* density_y, void* stream, FjErrorBuffer* error);

/* Carrier planes -> encoded output (monolithic carrier kernel, reference :1867). */
FjStatus fjb_render_carrier(FjbRecipe* recipe, const float* carrier_b, const float* carrier_g,
                            const float* carrier_r, ptrdiff_t carrier_stride, const float* src_alpha_source,
                            ptrdiff_t src_row_bytes, float* dst, ptrdiff_t dst_row_bytes, int32_t width,
                            int32_t height, uint32_t components, void* stream, FjErrorBuffer* error);

/* Capture density planes -> (print when the recipe's route prints) -> scan ->
 * encoded output (reference :2908 continue_from_capture_density + :2586 scan).
 * `src` supplies alpha when components == 4 (may be NULL: alpha 1). */
FjStatus fjb_render_from_density(FjbRecipe* recipe, const float* density_c, const float* density_m,
                                 const float* density_y, const float* src, ptrdiff_t src_row_bytes, float* dst,
                                 ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                 void* stream, FjErrorBuffer* error);

/* Scanner post effects (reference src/Cuda/Scan/JuicerCudaScanPipeline.cu:2982
 * juicer_cuda_print_focused_scan_linear_density_rgb + :2586-2878 launch_focused_scanner_post_output,
 * scheduled by src/Cuda/JuicerCudaExecutor.cpp:2384-2500): capture density planes ->
 * (print) -> scan to linear output RGB with the glare percent plane added in XYZ ->
 * lens blur -> unsharp mask -> encoded output. `post` is the prepared record
 * (active when its hash is non-zero); `glare_seed` and the glare origin (the frame's
 * source x1, y1) key the glare noise, see fjb_glare_seed. `scratch` holds
 * fjb_scanner_post_scratch_bytes(width, height) bytes of device memory. */
size_t fjb_scanner_post_scratch_bytes(int32_t width, int32_t height);
FjStatus fjb_render_from_density_post(FjbRecipe* recipe, const FjScannerPostEffects* post, uint64_t glare_seed,
                                      int32_t glare_origin_x, int32_t glare_origin_y, const float* density_c,
                                      const float* density_m, const float* density_y, const float* src,
                                      ptrdiff_t src_row_bytes, float* dst, ptrdiff_t dst_row_bytes, int32_t width,
                                      int32_t height, uint32_t components, float* scratch, size_t scratch_bytes,
                                      void* stream, FjErrorBuffer* error);

/* Film TC LUT on the device (reference rust/film-juicer-core/src/reconstruction.rs:594-677
 * build_tc_lut, which the reference runs on the host when a recipe is prepared): the
 * 192 x 192 x 81 spectra (`spectra`, device memory, [c][m][wavelength]) contracted with
 * the sensitivity into the R, G, B, +0 table (`table`, device memory, 192 * 192 * 4
 * floats, 16-byte aligned), word for word the reference's. method 0: Hanatos
 * irradiance, with the spectral blur when `spectral_blur` > 0 (radius up to 80
 * samples); method 2: Arctic reflectance relit by the reference illuminant and
 * normalised by the neutral response at the projected white; `apply_surface` (Hanatos)
 * multiplies by the surface correction of `surface_rgb` (host, 3 x 15);
 * `input_compression` remaps the table through the input gamut hull (`hull_xy`: host,
 * 1025 closed-polygon points; `hull_center`). The call allocates device memory for its
 * own use (256 B, plus 432 KiB with the surface correction and 864 KiB with the
 * compression), frees it and synchronises `stream` before returning. */
typedef struct FjbTcLutInput {
    const float* spectra;              /* device, 192*192*81 */
    const float* sensitivity_rgb;      /* host, 81 x 3 */
    const float* reference_illuminant; /* host, 81 */
    float projection_white_xyz[3];
    float spectral_blur;
    uint32_t method;
    uint32_t apply_surface;
    uint32_t input_compression;
    const float* surface_rgb;          /* host, 3 x 15, with apply_surface */
    const float* hull_xy;              /* host, 1025 x 2, with input_compression */
    float hull_center[2];
    uint32_t hull_available;
} FjbTcLutInput;
FjStatus fjb_tc_lut_build(const FjbTcLutInput* input, float* table, void* stream, FjErrorBuffer* error);

/* Output gamut boundary table on the device (reference rust/film-juicer-core/src/gamut.rs:760-829
 * build_output_boundary, run by the reference's host when a recipe is prepared): the
 * 64 x 720 maximum-chroma table of the OkLch output gamut compression (`cmax`, device
 * memory, 46 080 floats, lightness-major) for an output space given by its
 * OkLab-LMS-to-native-RGB matrix (`lms_to_native`, host, 3 x 3 FP64), word for word the
 * reference's. The call allocates device memory for its own use (12 KiB), frees it and
 * synchronises `stream` before returning. */
FjStatus fjb_gamut_boundary_build(const double* lms_to_native, float* cmax, void* stream, FjErrorBuffer* error);

/* Film and gate defects (reference src/Cuda/Scan/JuicerCudaScanPipeline.cu:2186-2242
 * juicer_cuda_apply_film_defects / juicer_cuda_build_gate_defect_transmittance_focused,
 * scheduled by src/Cuda/JuicerCudaExecutor.cpp:1674-1690, :2263-2279, :1806-1830).
 * `effects` is the prepared record; it must pass the reference's descriptor checks
 * (native/juicer_cuda_descriptors.cpp:467-515).
 * fjb_film_defects: film dust and scratches on capture density planes of a render
 *   window (full-frame pixel = pixel + the record's ROI offset): `dust` (width x height,
 *   required when film dust is on) receives the dust transmittance, and film scratches
 *   scale the three density planes.
 * fjb_gate_mask: gate dust x gate scratch transmittance, gate_width x gate_height.
 * `scratch` (may be null) holds the frame's particle table, fjb_film_defects_scratch_bytes
 *   / fjb_gate_mask_scratch_bytes bytes of device memory: every candidate particle is
 *   built once instead of once per tile that can reach it; without it (null or too
 *   small) the results are the same, computed more slowly.
 * fjb_render_from_density_effects: fjb_render_from_density_post with the defects'
 *   output effects: `dust` (or null) darkens the print exposure on the print route and
 *   the scanned XYZ on the direct route; with the gate output on, the weave resamples
 *   the linear planes and `gate_mask` (or null) multiplies them before encoding. */
size_t fjb_film_defects_scratch_bytes(const FjFilmEffects* effects, int32_t width, int32_t height);
size_t fjb_gate_mask_scratch_bytes(const FjFilmEffects* effects, int32_t gate_width, int32_t gate_height);
FjStatus fjb_film_defects(const FjFilmEffects* effects, int32_t width, int32_t height, float* density_c,
                          float* density_m, float* density_y, float* dust, void* scratch, size_t scratch_bytes,
                          void* stream, FjErrorBuffer* error);
FjStatus fjb_gate_mask(const FjFilmEffects* effects, float* gate_mask, int32_t gate_width, int32_t gate_height,
                       void* scratch, size_t scratch_bytes, void* stream, FjErrorBuffer* error);
FjStatus fjb_render_from_density_effects(FjbRecipe* recipe, const FjScannerPostEffects* post, uint64_t glare_seed,
                                         int32_t glare_origin_x, int32_t glare_origin_y,
                                         const FjFilmEffects* effects, const float* dust, const float* gate_mask,
                                         const float* density_c, const float* density_m, const float* density_y,
                                         const float* src, ptrdiff_t src_row_bytes, float* dst,
                                         ptrdiff_t dst_row_bytes, int32_t width, int32_t height, uint32_t components,
                                         float* scratch, size_t scratch_bytes, void* stream, FjErrorBuffer* error);

/* Glare seed of a frame (reference src/Cuda/JuicerCudaExecutor.cpp:2416, src/Hash.h:50):
 * FNV-1a 64 over the little-endian 8-byte words {recipe hash, frame token, source x1,
 * source y1}. */
uint64_t fjb_glare_seed(uint64_t recipe_hash, uint64_t frame_token, int32_t source_x1, int32_t source_y1);

/* Normalised Gaussian taps w[0..2 radius] (replaces the host preparation callback
 * FjHostPreparation.gaussian, native/juicer_cuda_call_scope.h:15, which the reference
 * serves from rust/film-juicer-core/src/optics/gaussian.rs:18-59): radius 1..2048,
 * sigma finite and positive; `count` >= 2 radius + 1. */
FjStatus fjb_gaussian_kernel_host(int32_t radius, float sigma_px, float* weights, size_t count,
                                  FjErrorBuffer* error);

/* Highlight reconstruction on the camera carrier planes B, G, R (reference
 * src/Cuda/Film/JuicerCudaHighlightBoost.cu:207-258 launch_highlight_boost; scheduled after
 * the camera exposure and before camera diffusion, src/Cuda/JuicerCudaExecutor.cpp:1155-1185).
 * `state` is fjb_highlight_boost_state_bytes() of device memory; the call is asynchronous.
 * fjb_highlight_boost_result synchronises `stream` and maps the disposition as the
 * reference does (src/ProcessRoot.cpp:4063-4096): applied / bypass succeed, an invalid
 * (negative or non-finite) carrier or a peak above FLT_MAX is FJ_STATUS_UNSUPPORTED_INPUT.
 * disposition: 0 bypass, 1 applied, 2 invalid carrier, 3 peak overflow. */
size_t fjb_highlight_boost_state_bytes(void);
FjStatus fjb_highlight_boost(const FjHighlightBoost* descriptor, float* carrier_b, float* carrier_g, float* carrier_r,
                             ptrdiff_t carrier_stride, int32_t width, int32_t height, void* state, void* stream,
                             FjErrorBuffer* error);
FjStatus fjb_highlight_boost_result(const void* state, void* stream, uint32_t* disposition, FjErrorBuffer* error);

/* Camera auto-exposure metering (reference src/Cuda/JuicerCudaAutoExposure.cu:314-520,
 * run by src/Cuda/JuicerCudaExecutor.cpp:1013 meter_camera_exposure). `src` points at
 * pixel (meter->source_bounds.x1, .y1). Writes the float exposure scale 2^-log2(Y) to
 * the device address `device_scale`; pass that address to
 * fjb_recipe_set_exposure_scale_device so later stages of the frame read it. Uses
 * scratch memory owned by the recipe, so calls on one recipe must not overlap.
 * FJ_METER_MEDIAN is rejected (FJ_STATUS_UNSUPPORTED_INPUT), as in the reference. */
FjStatus fjb_auto_exposure(FjbRecipe* recipe, const float* src, ptrdiff_t src_row_bytes, uint32_t components,
                           const FjAutoExposure* meter, float* device_scale, void* stream, FjErrorBuffer* error);

/* Bytes of device scratch fjb_scatter_halation needs for a width x height frame. */
size_t fjb_scatter_halation_scratch_bytes(int32_t width, int32_t height);

/* Emulsion scatter then halation back-reflection on the three carrier planes, in
 * place (reference src/Cuda/Film/JuicerCudaScatterHalation.cu:690
 * JuicerCuda::launch_scatter_halation). The descriptor's channels are R, G, B;
 * `stride` is in floats. `scratch` is caller-owned device memory of at least
 * fjb_scatter_halation_scratch_bytes(width, height) bytes. */
FjStatus fjb_scatter_halation(const FjScatterHalation* halation, float* carrier_r, float* carrier_g,
                              float* carrier_b, ptrdiff_t stride, int32_t width, int32_t height, float* scratch,
                              size_t scratch_bytes, void* stream, FjErrorBuffer* error);

/* Bytes of device scratch fjb_spatial_dir_build needs for a width x height frame. */
size_t fjb_spatial_dir_scratch_bytes(int32_t width, int32_t height);

/* Spatial DIR source + diffusion (reference src/Cuda/Film/JuicerCudaFilmPipeline.cu:1479
 * juicer_cuda_build_print_spatial_dir -> build_spatial_dir_impl :799). From the
 * carrier planes (when all three are given) or the source image it writes the
 * filtered donor-correction planes (Y, M, C receivers) and the raw log exposure (B,
 * G, R), all width x height floats. Operators: identity, reflect FIR (sigma < 3) and
 * the reflected-boundary recursive Gaussian (sigma >= 3), whose boundary weights are
 * derived on the host (see fjb_dir_boundary_host). Synchronises `stream`. */
FjStatus fjb_spatial_dir_build(FjbRecipe* recipe, const FjSpatialDir* spatial_dir, const float* src,
                               ptrdiff_t src_row_bytes, uint32_t components, const float* carrier_b,
                               const float* carrier_g, const float* carrier_r, ptrdiff_t carrier_stride,
                               int32_t width, int32_t height, float* filtered_y, float* filtered_m,
                               float* filtered_c, float* log_raw_b, float* log_raw_g, float* log_raw_r,
                               float* scratch, size_t scratch_bytes, void* stream, FjErrorBuffer* error);

/* The spatial DIR filter alone (the weighted Gaussian components of `spatial_dir`) on
 * three dense width x height planes Y, M, C, in -> out (distinct buffers). The
 * operator is linear and symmetric (half-sample reflected boundaries, symmetric
 * components), so it is also its own adjoint. `scratch` as for fjb_spatial_dir_build.
 * Synchronises `stream`. */
FjStatus fjb_spatial_dir_blur(const FjSpatialDir* spatial_dir, const float* in_y, const float* in_m,
                              const float* in_c, float* out_y, float* out_m, float* out_c, int32_t width,
                              int32_t height, float* scratch, size_t scratch_bytes, void* stream,
                              FjErrorBuffer* error);

/* The same filter prepared once for a frame size (its components' device tables), for
 * repeated use: fjb_spatial_dir_filter_apply only enqueues (dense width x height
 * planes, in -> out distinct, scratch as for fjb_spatial_dir_build);
 * fjb_spatial_dir_filter_destroy synchronises the device before it frees the tables. */
typedef struct FjbDirFilter FjbDirFilter;
FjStatus fjb_spatial_dir_filter_create(const FjSpatialDir* spatial_dir, int32_t width, int32_t height, void* stream,
                                       FjbDirFilter** out, FjErrorBuffer* error);
FjStatus fjb_spatial_dir_filter_apply(const FjbDirFilter* filter, const float* in_y, const float* in_m,
                                      const float* in_c, float* out_y, float* out_m, float* out_c, float* scratch,
                                      size_t scratch_bytes, void* stream, FjErrorBuffer* error);
void fjb_spatial_dir_filter_destroy(FjbDirFilter* filter);

/* Makes later capture-development calls on `recipe` use spatially filtered DIR
 * corrections and cached log exposure (all six device planes, or all NULL to return
 * to runtime DIR). */
FjStatus fjb_recipe_set_spatial_dir_planes(FjbRecipe* recipe, const float* filtered_y, const float* filtered_m,
                                           const float* filtered_c, const float* log_raw_b, const float* log_raw_g,
                                           const float* log_raw_r, FjErrorBuffer* error);

/* Reflected-boundary start weights (3 rows x *out_length, row-major) and end matrix
 * (*out_terminal_size squared, row-major) of one axis of a recursive DIR component;
 * the construction the reference obtains from its host through
 * native/juicer_dir_boundary_api.h:58-61 (fj_dir_boundary_acquire/view). */
FjStatus fjb_dir_boundary_host(const FjDirGaussian* component, int32_t axis_length, double* weights,
                               size_t weights_capacity, int32_t* out_length, int32_t* out_terminal_size,
                               double* terminal, FjErrorBuffer* error);

/* Nine exponential PSF components and their per-channel weights, as the host's
 * diffusion preparation produces them (reference native/juicer_diffusion_api.h:18-20,
 * fj_diffusion_components_prepare). */
typedef struct FjDiffusionComponents {
    double lambda_px[9];
    double red_weights[9];
    double green_weights[9];
    double blue_weights[9];
} FjDiffusionComponents;

/* Expands a diffusion filter record into its nine PSF components on the host (the
 * preparation the reference obtains from fj_diffusion_components_prepare,
 * native/juicer_diffusion_api.h:63). */
FjStatus fjb_diffusion_components_host(const FjDiffusion* diffusion, FjDiffusionComponents* out,
                                       FjErrorBuffer* error);

/* Camera or enlarger diffusion (reference src/Cuda/Diffusion/JuicerCudaDiffusion.cu:779
 * JuicerCuda::Diffusion::launch_stage): dst_c = (1 - f) src_c + f (PSF_c * src_c) with
 * PSF_c = sum_k w_ck exp(-rho / lambda_k) / (2 pi lambda_k^2) on the (2r+1)^2 grid,
 * normalised, and whole-sample reflection at the frame border. Planes R, G, B with
 * `stride` floats per row; dst must not alias src. radius_px <= 80. */
FjStatus fjb_diffusion(const FjDiffusionComponents* components, int32_t radius_px, double scatter_fraction,
                       const float* src_r, const float* src_g, const float* src_b, float* dst_r, float* dst_g,
                       float* dst_b, ptrdiff_t stride, int32_t width, int32_t height, void* stream,
                       FjErrorBuffer* error);

/* Same result as fjb_diffusion (to FP32 rounding of the PSF tables), for hosts that
 * cannot allocate device memory while rendering. No counterpart in the reference.
 * It allocates nothing: the PSF tables are built on the device into one static
 * device array of 3 x 81 x 176 floats (167 KiB) per device, and the call only
 * enqueues two kernels on `stream`, without synchronising. Limits: radius_px <= 80
 * (larger is rejected with FJ_STATUS_UNSUPPORTED_INPUT); weights finite and
 * non-negative, as fjb_diffusion_components_host produces them; the array is shared
 * by all calls on a device, so calls that may overlap (other streams or host threads)
 * race and must be ordered by the caller. The first call on each device looks up the
 * array's device address with that device current; make it before any stream
 * capture begins. That address is kept for the life of the process: do not reset the
 * device (cudaDeviceReset) between calls. */
FjStatus fjb_diffusion_no_alloc(const FjDiffusionComponents* components, int32_t radius_px, double scatter_fraction,
                                const float* src_r, const float* src_g, const float* src_b, float* dst_r,
                                float* dst_g, float* dst_b, ptrdiff_t stride, int32_t width, int32_t height,
                                void* stream, FjErrorBuffer* error);

/* Device copy of the static grain noise (blue-noise volume, Wang tiles and their
 * colour table), uploaded once and shared by every frame (the reference keeps the
 * same bytes resident, src/Cuda/JuicerCudaFilmPayloads.cpp:400-422). Synchronises
 * `stream`. */
typedef struct FjbNoise FjbNoise;
FjStatus fjb_noise_create(const FjStaticNoise* noise, void* stream, FjbNoise** out_noise, FjErrorBuffer* error);
FjStatus fjb_noise_destroy(FjbNoise* noise, FjErrorBuffer* error);

/* Bytes of device scratch fjb_visual_grain needs for a width x height frame. */
size_t fjb_visual_grain_scratch_bytes(int32_t width, int32_t height);

/* Density-space visual grain on the capture density planes C, M, Y in place
 * (reference src/Cuda/Scan/JuicerCudaScanPipeline.cu:3141 juicer_cuda_apply_visual_grain):
 * per channel up to three particle-size scales of Poisson particle samples (one layer
 * or three sublayers with dye-cloud blurs), correlation blurs, size-mix gain, shared
 * chroma mix, debug views. `noise` NULL draws from the Philox counter stream instead of
 * the blue noise. Sublayers read the recipe's density-layer curves. `scratch` is
 * caller-owned, 16-byte aligned, at least fjb_visual_grain_scratch_bytes bytes; calls
 * sharing a scratch buffer must not overlap. Does not synchronise. */
FjStatus fjb_visual_grain(FjbRecipe* recipe, const FjVisualGrain* grain, const FjbNoise* noise, float* density_c,
                          float* density_m, float* density_y, ptrdiff_t stride, int32_t width, int32_t height,
                          float* scratch, size_t scratch_bytes, void* stream, FjErrorBuffer* error);

/* Per-stage device time of fj_cuda_render frames (CUDA events recorded on the render
 * stream around each stage, read after the frame completes). Tracing aid; no
 * counterpart in the reference. */
#define FJB_STAGE_AUTO_EXPOSURE 0
#define FJB_STAGE_CAMERA_EXPOSURE 1
#define FJB_STAGE_CAMERA_DIFFUSION 2
#define FJB_STAGE_SCATTER_HALATION 3
#define FJB_STAGE_SPATIAL_DIR 4
#define FJB_STAGE_CAPTURE_DENSITY 5
#define FJB_STAGE_GRAIN 6
#define FJB_STAGE_PRINT_SCAN_OUTPUT 7
#define FJB_STAGE_MONOLITHIC 8
#define FJB_STAGE_FILM_DEFECTS 9
#define FJB_STAGE_ENLARGER_DIFFUSION 10
#define FJB_STAGE_COUNT 11
typedef struct FjbStageTimes {
    double total_ms[FJB_STAGE_COUNT];
    uint64_t frames[FJB_STAGE_COUNT];
} FjbStageTimes;
/* The print form (FJB_PRINT_*) of every recipe this owner renders, from the next
 * fj_cuda_render on. No counterpart in the reference. */
FjStatus fjb_owner_set_print_form(FjCuda* cuda, int32_t form, FjErrorBuffer* error);
/* Turns stage timing on (enable != 0) or off and resets the totals (single frames
 * through fj_cuda_render; batches are not timed per stage). */
FjStatus fjb_owner_stage_timing(FjCuda* cuda, int32_t enable, FjErrorBuffer* error);
/* Totals since the last fjb_owner_stage_timing call. */
FjStatus fjb_owner_stage_times(FjCuda* cuda, FjbStageTimes* out, FjErrorBuffer* error);

/* Batches of frames (no counterpart in the reference, which renders one frame per
 * fj_cuda_render call). fjb_render_batch renders `count` frames -- any mix of sizes,
 * stocks, papers and stage sets, each checked as fj_cuda_render checks it -- in order
 * on `stream` (the frames' own stream fields are ignored), with one read-back of all
 * frames' flag words at the end instead of one host round trip per frame.
 * outcomes[i] is frame i's FjRenderOutcome; the return value is the first failing
 * frame's status (no work is enqueued when a frame fails its checks).
 *
 * graph_token != 0 (and a non-null stream, and every frame with a non-zero
 * recipe_hash): after the call's own eager render, the batch's work (every launch,
 * flag copy and the read-back) is captured into a CUDA graph kept by the owner under
 * that token. A later call with the same token and frame count replays the graph in
 * one launch: the caller guarantees that the frames' buffers and descriptors are the
 * ones of the captured call (pixel contents may change). A new token recaptures; the
 * owner drops the graph whenever a buffer it references is regrown or freed.
 * submissions may be null (frame tokens 0). */
FjStatus fjb_render_batch(FjCuda* cuda, const FjCudaContext* context, const FjFrame* frames,
                          const FjSubmission* submissions, const FjPreparedHostData* const* prepared, int32_t count,
                          void* stream, uint64_t graph_token, FjRenderOutcome* outcomes, FjErrorBuffer* error);
/* Diffusion form autotuning (no counterpart in the reference): with enable != 0 the
 * owner times the direct and the FFT form of camera and enlarger diffusion on the
 * first frame of each (width, height, radius) and keeps the faster; off (the default),
 * the fixed size rule chooses. fjb_owner_diffusion_form reports the decision
 * (FJB_DIFFUSION_*, -1 undecided). */
#define FJB_DIFFUSION_DIRECT 0
#define FJB_DIFFUSION_FFT 1
FjStatus fjb_owner_set_autotune(FjCuda* cuda, int32_t enable, FjErrorBuffer* error);
FjStatus fjb_owner_diffusion_form(FjCuda* cuda, int32_t width, int32_t height, int32_t radius_px, int32_t* form,
                                  FjErrorBuffer* error);

/* Kernel launches this library has made in the process so far (all entry points). */
uint64_t fjb_kernel_launches(void);

/* Scanner LUT input record (reference native/juicer_cuda_frame_values.h FjScannerLutInput). */
typedef struct FjbScannerLutInput {
    FjFloatSpan eps_c, eps_m, eps_y;
    FjFloatSpan weighted_x, weighted_y, weighted_z, baseline_min;
    float range_min_cmy[3], inverse_span_cmy[3];
    int32_t sample_count;
    float inv_yn;
    uint32_t has_baseline, medium, resolution;
} FjbScannerLutInput;

/* Builds the six scanner PCHIP arrays on the device (FP64) and copies them into the
 * caller's HOST buffers: log2_xyz/slope_c/slope_m/slope_y hold 3*r^3 floats,
 * cell_min/cell_max 3*(r-1)^3. Synchronous. Replaces the Rust host build
 * rust/film-juicer-core/src/scanner/lut.rs:187 behind the callback
 * native/juicer_cuda_call_scope.h:14. */
FjStatus fjb_scanner_lut_build_host(const FjbScannerLutInput* input, float* log2_xyz, float* slope_c,
                                    float* slope_m, float* slope_y, float* cell_min, float* cell_max,
                                    FjErrorBuffer* error);

#ifdef __cplusplus
}
#endif

#endif /* JUICER_B200_H */
