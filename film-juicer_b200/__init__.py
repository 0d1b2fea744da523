"""film-juicer-b200: B200-native render path of Film-Juicer's film-process model.

The product is libjuicer_b200.so (CUDA for sm_100a behind the C-ABI in
include/juicer_cuda_api.h and include/juicer_b200.h). This package loads it and
mirrors the reference host's records (abi.py), prepares recipes from profiles
(prepare.py) and offers thin Python calls over the C-ABI (runtime.py). There is no
CPU render path: every render call goes through the CUDA library and fails loudly
when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjuicer_b200.so")

_lib = None

_EXPORTS = {
    "fj_cuda_create": (abi.FjStatus, [C.POINTER(C.c_void_p), C.POINTER(abi.FjErrorBuffer)]),
    "fjb_scanner_post_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
    "fjb_render_from_density_post": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjScannerPostEffects), C.c_uint64,
                                                    C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_ssize_t, C.c_void_p, C.c_ssize_t, C.c_int32,
                                                    C.c_int32, C.c_uint32, C.c_void_p, C.c_size_t, C.c_void_p,
                                                    C.POINTER(abi.FjErrorBuffer)]),
    "fjb_glare_seed": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_int32, C.c_int32]),
    "fjb_gamut_boundary_build": (abi.FjStatus, [C.POINTER(C.c_double), C.c_void_p, C.c_void_p,
                                                C.POINTER(abi.FjErrorBuffer)]),
    "fjb_tc_lut_build": (abi.FjStatus, [C.POINTER(abi.FjbTcLutInput), C.c_void_p, C.c_void_p,
                                        C.POINTER(abi.FjErrorBuffer)]),
    "fjb_film_defects_scratch_bytes": (C.c_size_t, [C.POINTER(abi.FjFilmEffects), C.c_int32, C.c_int32]),
    "fjb_gate_mask_scratch_bytes": (C.c_size_t, [C.POINTER(abi.FjFilmEffects), C.c_int32, C.c_int32]),
    "fjb_film_defects": (abi.FjStatus, [C.POINTER(abi.FjFilmEffects), C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                        C.POINTER(abi.FjErrorBuffer)]),
    "fjb_gate_mask": (abi.FjStatus, [C.POINTER(abi.FjFilmEffects), C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                     C.c_size_t, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_render_from_density_effects": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjScannerPostEffects), C.c_uint64,
                                                       C.c_int32, C.c_int32, C.POINTER(abi.FjFilmEffects),
                                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.c_void_p, C.c_ssize_t, C.c_void_p, C.c_ssize_t, C.c_int32,
                                                       C.c_int32, C.c_uint32, C.c_void_p, C.c_size_t, C.c_void_p,
                                                       C.POINTER(abi.FjErrorBuffer)]),
    "fjb_highlight_boost_state_bytes": (C.c_size_t, []),
    "fjb_highlight_boost": (abi.FjStatus, [C.POINTER(abi.FjHighlightBoost), C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_ssize_t, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                           C.POINTER(abi.FjErrorBuffer)]),
    "fjb_highlight_boost_result": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32),
                                                  C.POINTER(abi.FjErrorBuffer)]),
    "fjb_gaussian_kernel_host": (abi.FjStatus, [C.c_int32, C.c_float, C.POINTER(C.c_float), C.c_size_t,
                                                C.POINTER(abi.FjErrorBuffer)]),
    "fj_cuda_check_terminal": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fj_cuda_inspect": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjFrame), C.POINTER(abi.FjCudaContext),
                                       C.POINTER(abi.FjErrorBuffer)]),
    "fj_cuda_render": (abi.FjRenderOutcome, [C.c_void_p, C.POINTER(abi.FjCudaContext), C.POINTER(abi.FjFrame),
                                             C.POINTER(abi.FjSubmission), C.POINTER(abi.FjPreparedHostData),
                                             abi.FjAbortCallback, C.POINTER(abi.FjErrorBuffer)]),
    "fj_cuda_retire_instance": (abi.FjStatus, [C.c_void_p, C.c_uint64, C.POINTER(abi.FjErrorBuffer)]),
    "fj_cuda_shutdown": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fj_cuda_destroy": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_recipe_create": (abi.FjStatus, [C.POINTER(abi.FjPreparedHostData), C.c_void_p, C.POINTER(C.c_void_p),
                                         C.POINTER(abi.FjErrorBuffer)]),
    "fjb_recipe_destroy": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_recipe_set_exposure_scale_device": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_recipe_clear_flags": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_recipe_set_print_form": (abi.FjStatus, [C.c_void_p, C.c_int32, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_render_batch": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjCudaContext), C.POINTER(abi.FjFrame),
                                        C.POINTER(abi.FjSubmission), C.POINTER(C.c_void_p), C.c_int32, C.c_void_p,
                                        C.c_uint64, C.POINTER(abi.FjRenderOutcome), C.POINTER(abi.FjErrorBuffer)]),
    "fjb_owner_set_autotune": (abi.FjStatus, [C.c_void_p, C.c_int32, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_owner_diffusion_form": (abi.FjStatus, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                                C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_defaults": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams), C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_forward": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams), C.c_void_p, C.c_ssize_t, C.c_uint32,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                       C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_scratch_bytes": (C.c_size_t, []),
    "fjb_fit_forward_carrier": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams), C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_ssize_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                               C.c_int32, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_vjp_carrier": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams), C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_ssize_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                           C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_size_t, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_dir_source_carrier": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams)] + [C.c_void_p] * 3 +
                                   [C.c_ssize_t] + [C.c_void_p] * 3 + [C.c_int32, C.c_int32, C.c_void_p,
                                                                     C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_forward_spatial_carrier": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams)] + [C.c_void_p] * 3 +
                                        [C.c_ssize_t] + [C.c_void_p] * 6 + [C.c_int32, C.c_int32, C.c_void_p,
                                                                          C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_vjp_spatial_carrier": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams)] + [C.c_void_p] * 3 +
                                    [C.c_ssize_t] + [C.c_void_p] * 6 + [C.c_int32, C.c_int32] + [C.c_void_p] * 8 +
                                    [C.c_size_t, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_dir_source_vjp_carrier": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams)] + [C.c_void_p] * 3 +
                                       [C.c_ssize_t] + [C.c_void_p] * 3 + [C.c_int32, C.c_int32] +
                                       [C.c_void_p] * 5 + [C.c_size_t, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_fit_vjp": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbFitParams), C.c_void_p, C.c_ssize_t, C.c_uint32,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                   C.c_size_t, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_enlarger_linear_exposure": (abi.FjStatus, [C.c_void_p] + [C.c_void_p] * 7 + [C.c_int32, C.c_int32, C.c_void_p,
                                                                                       C.POINTER(abi.FjErrorBuffer)]),
    "fjb_enlarger_develop": (abi.FjStatus, [C.c_void_p] + [C.c_void_p] * 6 + [C.c_int32, C.c_int32, C.c_void_p,
                                                                               C.POINTER(abi.FjErrorBuffer)]),
    "fjb_render_from_print_density": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                      C.c_ssize_t, C.c_void_p, C.c_ssize_t, C.c_int32, C.c_int32,
                                                      C.c_uint32, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_print_raw": (abi.FjStatus, [C.c_void_p] + [C.c_void_p] * 6 + [C.c_int32, C.c_int32, C.c_void_p,
                                                                        C.POINTER(abi.FjErrorBuffer)]),
    "fjb_recipe_read_flags": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32),
                                             C.POINTER(abi.FjErrorBuffer)]),
    "fjb_render_pixels": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.c_ssize_t, C.c_void_p, C.c_ssize_t, C.c_int32,
                                         C.c_int32, C.c_uint32, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_camera_exposure": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.c_ssize_t, C.c_uint32, C.c_int32, C.c_int32,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_ssize_t, C.c_void_p,
                                           C.POINTER(abi.FjErrorBuffer)]),
    "fjb_capture_density": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.c_ssize_t, C.c_uint32, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_ssize_t, C.c_int32, C.c_int32, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_render_carrier": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_ssize_t,
                                          C.c_void_p, C.c_ssize_t, C.c_void_p, C.c_ssize_t, C.c_int32, C.c_int32,
                                          C.c_uint32, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_render_from_density": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_ssize_t, C.c_void_p, C.c_ssize_t, C.c_int32, C.c_int32,
                                               C.c_uint32, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_auto_exposure": (abi.FjStatus, [C.c_void_p, C.c_void_p, C.c_ssize_t, C.c_uint32, C.POINTER(abi.FjAutoExposure),
                                         C.c_void_p, C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_scatter_halation_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
    "fjb_scatter_halation": (abi.FjStatus, [C.POINTER(abi.FjScatterHalation), C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_ssize_t, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p,
                                            C.POINTER(abi.FjErrorBuffer)]),
    "fjb_spatial_dir_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
    "fjb_spatial_dir_build": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjSpatialDir), C.c_void_p, C.c_ssize_t,
                                             C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_ssize_t, C.c_int32,
                                             C.c_int32] + [C.c_void_p] * 7 + [C.c_size_t, C.c_void_p,
                                                                                C.POINTER(abi.FjErrorBuffer)]),
    "fjb_spatial_dir_blur": (abi.FjStatus, [C.POINTER(abi.FjSpatialDir)] + [C.c_void_p] * 6 +
                             [C.c_int32, C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p,
                              C.POINTER(abi.FjErrorBuffer)]),
    "fjb_spatial_dir_filter_create": (abi.FjStatus, [C.POINTER(abi.FjSpatialDir), C.c_int32, C.c_int32, C.c_void_p,
                                                     C.POINTER(C.c_void_p), C.POINTER(abi.FjErrorBuffer)]),
    "fjb_spatial_dir_filter_apply": (abi.FjStatus, [C.c_void_p] * 7 + [C.c_void_p, C.c_size_t, C.c_void_p,
                                                                       C.POINTER(abi.FjErrorBuffer)]),
    "fjb_spatial_dir_filter_destroy": (None, [C.c_void_p]),
    "fjb_recipe_set_spatial_dir_planes": (abi.FjStatus, [C.c_void_p] + [C.c_void_p] * 6 +
                                          [C.POINTER(abi.FjErrorBuffer)]),
    "fjb_dir_boundary_host": (abi.FjStatus, [C.POINTER(abi.FjDirGaussian), C.c_int32, C.POINTER(C.c_double),
                                             C.c_size_t, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                             C.POINTER(C.c_double), C.POINTER(abi.FjErrorBuffer)]),
    "fjb_diffusion_components_host": (abi.FjStatus, [C.POINTER(abi.FjDiffusion), C.POINTER(abi.FjDiffusionComponents),
                                                     C.POINTER(abi.FjErrorBuffer)]),
    "fjb_diffusion": (abi.FjStatus, [C.POINTER(abi.FjDiffusionComponents), C.c_int32, C.c_double] +
                      [C.c_void_p] * 6 + [C.c_ssize_t, C.c_int32, C.c_int32, C.c_void_p,
                                          C.POINTER(abi.FjErrorBuffer)]),
    "fjb_diffusion_no_alloc": (abi.FjStatus, [C.POINTER(abi.FjDiffusionComponents), C.c_int32, C.c_double] +
                               [C.c_void_p] * 6 + [C.c_ssize_t, C.c_int32, C.c_int32, C.c_void_p,
                                                   C.POINTER(abi.FjErrorBuffer)]),
    "fjb_noise_create": (abi.FjStatus, [C.POINTER(abi.FjStaticNoise), C.c_void_p, C.POINTER(C.c_void_p),
                                        C.POINTER(abi.FjErrorBuffer)]),
    "fjb_noise_destroy": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_visual_grain_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
    "fjb_visual_grain": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjVisualGrain), C.c_void_p] + [C.c_void_p] * 3 +
                         [C.c_ssize_t, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p,
                          C.POINTER(abi.FjErrorBuffer)]),
    "fjb_owner_stage_timing": (abi.FjStatus, [C.c_void_p, C.c_int32, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_owner_set_print_form": (abi.FjStatus, [C.c_void_p, C.c_int32, C.POINTER(abi.FjErrorBuffer)]),
    "fjb_owner_stage_times": (abi.FjStatus, [C.c_void_p, C.POINTER(abi.FjbStageTimes), C.POINTER(abi.FjErrorBuffer)]),
    "fjb_kernel_launches": (C.c_uint64, []),
    "fjb_scanner_lut_build_host": (abi.FjStatus, [C.POINTER(abi.FjbScannerLutInput)] + [C.c_void_p] * 6 +
                                   [C.POINTER(abi.FjErrorBuffer)]),
}


def exported_names() -> list[str]:
    return list(_EXPORTS)


def load_library(path: str | None = None):
    """Loads libjuicer_b200.so and declares every exported signature. Raises if missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libjuicer_b200.so is not built ({p}); run __graft_entry__.build()")
    lib = C.CDLL(p)
    for name, (res, args) in _EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
