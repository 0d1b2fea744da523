"""Python calls over the C-ABI of libjuicer_b200.so.

torch supplies device memory and streams here (plumbing only); every pixel is
computed by the CUDA library. Nothing in this module has a CPU fallback: without the
library or a GPU it raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, load_library


class FjError(RuntimeError):
    def __init__(self, where: str, status, text: str):
        super().__init__(f"{where}: status category {status.category} (api {status.api}, code "
                         f"{status.native_code}): {text}")
        self.status = status


def _check(where: str, status, err: abi.ErrorText):
    if status.category != abi.FJ_STATUS_SUCCESS:
        raise FjError(where, status, err.text)


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("CUDA device required: the render path has no CPU implementation")
    return torch


def _ptr(t) -> int:
    return int(t.data_ptr())


def _stream_handle(stream) -> int:
    return int(stream.cuda_stream) if stream is not None else 0


class DeviceRecipe:
    """Device tables of one prepared recipe (fjb_recipe_create / fjb_recipe_destroy)."""

    def __init__(self, record, stream=None):
        self.lib = load_library()
        self.record = record
        self.handle = C.c_void_p()
        err = abi.ErrorText()
        st = self.lib.fjb_recipe_create(record.pointer(), C.c_void_p(_stream_handle(stream)),
                                        C.byref(self.handle), C.byref(err.buf))
        _check("fjb_recipe_create", st, err)

    def close(self):
        if self.handle:
            err = abi.ErrorText()
            self.lib.fjb_recipe_destroy(self.handle, C.byref(err.buf))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_print_form(self, form: int):
        """abi.FJB_PRINT_FP32 | FJB_PRINT_TENSOR | FJB_PRINT_TENSOR_SPLIT."""
        err = abi.ErrorText()
        _check("fjb_recipe_set_print_form", self.lib.fjb_recipe_set_print_form(self.handle, form, C.byref(err.buf)),
               err)

    def print_raw(self, density, raw, stream=None):
        """The print's spectral integral (C, M, Y planes) of density planes (C, M, Y)."""
        c, m, y = density
        h, w = c.shape
        err = abi.ErrorText()
        st = self.lib.fjb_print_raw(self.handle, *[C.c_void_p(_ptr(t)) for t in (c, m, y, *raw)], w, h,
                                    C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
        _check("fjb_print_raw", st, err)

    def enlarger_linear_exposure(self, density, linear, dust=None, stream=None):
        """Print-linear exposure planes (C-, M-, Y-forming) of capture density planes."""
        c, m, y = density
        h, w = c.shape
        err = abi.ErrorText()
        st = self.lib.fjb_enlarger_linear_exposure(self.handle, *[C.c_void_p(_ptr(t)) for t in (c, m, y)],
                                                   C.c_void_p(_ptr(dust) if dust is not None else 0),
                                                   *[C.c_void_p(_ptr(t)) for t in linear], w, h,
                                                   C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
        _check("fjb_enlarger_linear_exposure", st, err)

    def enlarger_develop(self, linear, density, stream=None):
        """Print density planes C, M, Y of (diffused) print-linear exposure planes."""
        h, w = linear[0].shape
        err = abi.ErrorText()
        st = self.lib.fjb_enlarger_develop(self.handle, *[C.c_void_p(_ptr(t)) for t in (*linear, *density)], w, h,
                                           C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
        _check("fjb_enlarger_develop", st, err)

    def render_from_print_density(self, density, src, dst, stream=None):
        c, m, y = density
        h, w, comps = dst.shape
        err = abi.ErrorText()
        st = self.lib.fjb_render_from_print_density(self.handle, C.c_void_p(_ptr(c)), C.c_void_p(_ptr(m)),
                                                    C.c_void_p(_ptr(y)), C.c_void_p(_ptr(src) if src is not None else 0),
                                                    (src.stride(0) * 4) if src is not None else 0, C.c_void_p(_ptr(dst)),
                                                    dst.stride(0) * 4, w, h, comps, C.c_void_p(_stream_handle(stream)),
                                                    C.byref(err.buf))
        _check("fjb_render_from_print_density", st, err)

    def set_exposure_scale_device(self, tensor):
        err = abi.ErrorText()
        st = self.lib.fjb_recipe_set_exposure_scale_device(self.handle, C.c_void_p(_ptr(tensor) if tensor is not None
                                                                                    else 0), C.byref(err.buf))
        _check("fjb_recipe_set_exposure_scale_device", st, err)

    def clear_flags(self, stream=None):
        err = abi.ErrorText()
        _check("fjb_recipe_clear_flags",
               self.lib.fjb_recipe_clear_flags(self.handle, C.c_void_p(_stream_handle(stream)), C.byref(err.buf)), err)

    def read_flags(self, stream=None) -> int:
        err = abi.ErrorText()
        v = C.c_uint32()
        _check("fjb_recipe_read_flags", self.lib.fjb_recipe_read_flags(
            self.handle, C.c_void_p(_stream_handle(stream)), C.byref(v), C.byref(err.buf)), err)
        return int(v.value)

    def render(self, src, dst, stream=None):
        """src/dst: contiguous float32 CUDA tensors of shape (H, W, 3|4)."""
        h, w, comps = src.shape
        err = abi.ErrorText()
        st = self.lib.fjb_render_pixels(self.handle, C.c_void_p(_ptr(src)), src.stride(0) * 4,
                                        C.c_void_p(_ptr(dst)), dst.stride(0) * 4, w, h, comps,
                                        C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
        _check("fjb_render_pixels", st, err)

    def camera_exposure(self, src, planes, stream=None):
        h, w, comps = src.shape
        b, g, r = planes
        err = abi.ErrorText()
        st = self.lib.fjb_camera_exposure(self.handle, C.c_void_p(_ptr(src)), src.stride(0) * 4, comps, w, h,
                                          C.c_void_p(_ptr(b)), C.c_void_p(_ptr(g)), C.c_void_p(_ptr(r)),
                                          b.stride(0), C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
        _check("fjb_camera_exposure", st, err)

    def capture_density(self, src, density, carrier=None, stream=None):
        c, m, y = density
        h, w = c.shape
        comps = src.shape[2] if src is not None else 3
        cb, cg, cr = carrier if carrier is not None else (None, None, None)
        err = abi.ErrorText()
        st = self.lib.fjb_capture_density(
            self.handle, C.c_void_p(_ptr(src) if src is not None else 0), (src.stride(0) * 4) if src is not None else 0,
            comps, C.c_void_p(_ptr(cb) if cb is not None else 0), C.c_void_p(_ptr(cg) if cg is not None else 0),
            C.c_void_p(_ptr(cr) if cr is not None else 0), cb.stride(0) if cb is not None else 0, w, h,
            C.c_void_p(_ptr(c)), C.c_void_p(_ptr(m)), C.c_void_p(_ptr(y)), C.c_void_p(_stream_handle(stream)),
            C.byref(err.buf))
        _check("fjb_capture_density", st, err)

    def render_carrier(self, carrier, src, dst, stream=None):
        b, g, r = carrier
        h, w, comps = dst.shape
        err = abi.ErrorText()
        st = self.lib.fjb_render_carrier(self.handle, C.c_void_p(_ptr(b)), C.c_void_p(_ptr(g)), C.c_void_p(_ptr(r)),
                                         b.stride(0), C.c_void_p(_ptr(src) if src is not None else 0),
                                         (src.stride(0) * 4) if src is not None else 0, C.c_void_p(_ptr(dst)),
                                         dst.stride(0) * 4, w, h, comps, C.c_void_p(_stream_handle(stream)),
                                         C.byref(err.buf))
        _check("fjb_render_carrier", st, err)

    def render_from_density(self, density, src, dst, stream=None):
        c, m, y = density
        h, w, comps = dst.shape
        err = abi.ErrorText()
        st = self.lib.fjb_render_from_density(self.handle, C.c_void_p(_ptr(c)), C.c_void_p(_ptr(m)),
                                              C.c_void_p(_ptr(y)), C.c_void_p(_ptr(src) if src is not None else 0),
                                              (src.stride(0) * 4) if src is not None else 0, C.c_void_p(_ptr(dst)),
                                              dst.stride(0) * 4, w, h, comps, C.c_void_p(_stream_handle(stream)),
                                              C.byref(err.buf))
        _check("fjb_render_from_density", st, err)


    def set_spatial_dir_planes(self, filtered=None, log_raw=None):
        """Capture development reads these planes (filtered Y, M, C; log raw B, G, R)
        from now on; None returns to runtime DIR."""
        ptrs = [C.c_void_p(_ptr(t)) for t in (*filtered, *log_raw)] if filtered is not None else [C.c_void_p(0)] * 6
        err = abi.ErrorText()
        _check("fjb_recipe_set_spatial_dir_planes",
               self.lib.fjb_recipe_set_spatial_dir_planes(self.handle, *ptrs, C.byref(err.buf)), err)

    def spatial_dir_build(self, spatial_dir, filtered, log_raw, *, src=None, carrier=None, scratch=None,
                          stream=None):
        """Spatial-DIR source + diffusion into `filtered` (Y, M, C) and `log_raw` (B, G, R)."""
        torch = _torch()
        h, w = filtered[0].shape
        need = int(self.lib.fjb_spatial_dir_scratch_bytes(w, h))
        if scratch is None:
            scratch = torch.empty(need // 4, dtype=torch.float32, device=filtered[0].device)
        cb, cg, cr = carrier if carrier is not None else (None, None, None)
        err = abi.ErrorText()
        st = self.lib.fjb_spatial_dir_build(
            self.handle, C.byref(spatial_dir), C.c_void_p(_ptr(src) if src is not None else 0),
            (src.stride(0) * 4) if src is not None else 0, src.shape[2] if src is not None else 3,
            C.c_void_p(_ptr(cb) if cb is not None else 0), C.c_void_p(_ptr(cg) if cg is not None else 0),
            C.c_void_p(_ptr(cr) if cr is not None else 0), cb.stride(0) if cb is not None else 0, w, h,
            *[C.c_void_p(_ptr(t)) for t in (*filtered, *log_raw)], C.c_void_p(_ptr(scratch)), scratch.numel() * 4,
            C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
        _check("fjb_spatial_dir_build", st, err)
        return scratch


def render_pixels_numpy(record, src: np.ndarray) -> np.ndarray:
    """One fused per-pixel render of a host image (H, W, 3|4) through the C-ABI."""
    torch = _torch()
    rec = DeviceRecipe(record)
    s = torch.from_numpy(np.ascontiguousarray(src, dtype=np.float32)).cuda()
    d = torch.empty_like(s)
    rec.render(s, d)
    torch.cuda.synchronize()
    out = d.cpu().numpy()
    rec.close()
    return out


def scanner_lut_build_host(inp: "abi.FjbScannerLutInput"):
    """Six scanner PCHIP arrays built on the device (FP64) and returned as numpy arrays."""
    lib = load_library()
    r = int(inp.resolution)
    nodes, cells = 3 * r ** 3, 3 * (r - 1) ** 3
    outs = [np.zeros(nodes, np.float32) for _ in range(4)] + [np.zeros(cells, np.float32) for _ in range(2)]
    err = abi.ErrorText()
    st = lib.fjb_scanner_lut_build_host(C.byref(inp), *[C.c_void_p(o.ctypes.data) for o in outs], C.byref(err.buf))
    _check("fjb_scanner_lut_build_host", st, err)
    return outs


def meter_record(width: int, height: int, *, method: int = 0, preview: tuple[int, int] | None = None,
                 meter: tuple[int, int, int, int] | None = None) -> "abi.FjAutoExposure":
    """FjAutoExposure over a width x height source (preview long edge <= 256, as the host uses)."""
    m = abi.FjAutoExposure()
    m.source_bounds = abi.FjRect(0, 0, width, height)
    mx1, my1, mx2, my2 = meter if meter is not None else (0, 0, width, height)
    m.meter_bounds = abi.FjRect(mx1, my1, mx2, my2)
    if preview is None:
        mw, mh = mx2 - mx1, my2 - my1
        s = min(1.0, 256.0 / max(mw, mh))
        preview = (max(1, int(round(mw * s))), max(1, int(round(mh * s))))
    m.preview_width, m.preview_height = preview
    m.method = method
    m.hash = 1
    return m


def auto_exposure(recipe: "DeviceRecipe", src, meter: "abi.FjAutoExposure", scale_out, stream=None):
    """Meters `src` (CUDA tensor H x W x comps) into the device float `scale_out`."""
    err = abi.ErrorText()
    st = recipe.lib.fjb_auto_exposure(recipe.handle, C.c_void_p(_ptr(src)), src.stride(0) * 4, src.shape[2],
                                      C.byref(meter), C.c_void_p(_ptr(scale_out)), C.c_void_p(_stream_handle(stream)),
                                      C.byref(err.buf))
    _check("fjb_auto_exposure", st, err)


def spatial_dir_blur(spatial_dir: "abi.FjSpatialDir", planes_ymc, out_ymc, stream=None, scratch=None):
    """fjb_spatial_dir_blur: the spatial DIR filter of three dense (H, W) float32 CUDA
    planes (Y, M, C) into `out_ymc`; returns the scratch for reuse."""
    torch = _torch()
    lib = load_library()
    h, w = planes_ymc[0].shape
    for t in (*planes_ymc, *out_ymc):
        if not t.is_contiguous() or tuple(t.shape) != (h, w):
            raise ValueError("spatial DIR blur planes must be dense (H, W) tensors of one size")
    need = int(lib.fjb_spatial_dir_scratch_bytes(w, h))
    if scratch is None or scratch.numel() * 4 < need:
        scratch = torch.empty(need // 4 + 1, dtype=torch.float32, device=planes_ymc[0].device)
    err = abi.ErrorText()
    st = lib.fjb_spatial_dir_blur(C.byref(spatial_dir), *[C.c_void_p(_ptr(t)) for t in (*planes_ymc, *out_ymc)], w, h,
                                  C.c_void_p(_ptr(scratch)), scratch.numel() * 4, C.c_void_p(_stream_handle(stream)),
                                  C.byref(err.buf))
    _check("fjb_spatial_dir_blur", st, err)
    return scratch


class DirFilter:
    """A spatial DIR filter prepared once for a frame size (fjb_spatial_dir_filter_*);
    `apply` enqueues it on three dense (H, W) planes (Y, M, C)."""

    def __init__(self, spatial_dir: "abi.FjSpatialDir", width: int, height: int, stream=None):
        self.lib = load_library()
        self.width, self.height = width, height
        self.handle = C.c_void_p()
        self.scratch = None
        err = abi.ErrorText()
        _check("fjb_spatial_dir_filter_create",
               self.lib.fjb_spatial_dir_filter_create(C.byref(spatial_dir), width, height,
                                                      C.c_void_p(_stream_handle(stream)), C.byref(self.handle),
                                                      C.byref(err.buf)), err)

    def apply(self, planes_ymc, out_ymc, stream=None):
        torch = _torch()
        for t in (*planes_ymc, *out_ymc):
            if not t.is_contiguous() or tuple(t.shape) != (self.height, self.width):
                raise ValueError("spatial DIR filter planes must be dense (H, W) tensors of the filter's size")
        need = int(self.lib.fjb_spatial_dir_scratch_bytes(self.width, self.height))
        if self.scratch is None or self.scratch.numel() * 4 < need:
            self.scratch = torch.empty(need // 4 + 1, dtype=torch.float32, device=planes_ymc[0].device)
        err = abi.ErrorText()
        _check("fjb_spatial_dir_filter_apply",
               self.lib.fjb_spatial_dir_filter_apply(self.handle, *[C.c_void_p(_ptr(t)) for t in (*planes_ymc, *out_ymc)],
                                                     C.c_void_p(_ptr(self.scratch)), self.scratch.numel() * 4,
                                                     C.c_void_p(_stream_handle(stream)), C.byref(err.buf)), err)
        return out_ymc

    def close(self):
        if self.handle:
            self.lib.fjb_spatial_dir_filter_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scatter_halation(descriptor: "abi.FjScatterHalation", planes_rgb, stream=None, scratch=None):
    """In-place scatter/halation on three CUDA planes (R, G, B), each (H, W) float32."""
    torch = _torch()
    lib = load_library()
    r, g, b = planes_rgb
    h, w = r.shape
    need = int(lib.fjb_scatter_halation_scratch_bytes(w, h))
    if scratch is None:
        scratch = torch.empty(need // 4, dtype=torch.float32, device=r.device)
    err = abi.ErrorText()
    st = lib.fjb_scatter_halation(C.byref(descriptor), C.c_void_p(_ptr(r)), C.c_void_p(_ptr(g)), C.c_void_p(_ptr(b)),
                                  r.stride(0), w, h, C.c_void_p(_ptr(scratch)), scratch.numel() * 4,
                                  C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_scatter_halation", st, err)
    return scratch


def diffusion_components(diffusion: "abi.FjDiffusion") -> "abi.FjDiffusionComponents":
    """The nine PSF components of a diffusion record (host computation in the library)."""
    lib = load_library()
    out = abi.FjDiffusionComponents()
    err = abi.ErrorText()
    _check("fjb_diffusion_components_host", lib.fjb_diffusion_components_host(C.byref(diffusion), C.byref(out),
                                                                              C.byref(err.buf)), err)
    return out


def diffusion(components, radius: int, fraction: float, src_rgb, dst_rgb, stream=None):
    """dst = (1 - f) src + f (PSF * src) for three CUDA planes (R, G, B)."""
    lib = load_library()
    err = abi.ErrorText()
    h, w = src_rgb[0].shape
    st = lib.fjb_diffusion(C.byref(components), radius, fraction, *[C.c_void_p(_ptr(t)) for t in src_rgb],
                           *[C.c_void_p(_ptr(t)) for t in dst_rgb], src_rgb[0].stride(0), w, h,
                           C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_diffusion", st, err)


class DeviceNoise:
    """Device copy of the static grain noise (fjb_noise_create / fjb_noise_destroy)."""

    def __init__(self, noise_record, stream=None):
        self.lib = load_library()
        self.handle = C.c_void_p()
        err = abi.ErrorText()
        _check("fjb_noise_create", self.lib.fjb_noise_create(C.byref(noise_record), C.c_void_p(_stream_handle(stream)),
                                                             C.byref(self.handle), C.byref(err.buf)), err)

    def close(self):
        if self.handle:
            err = abi.ErrorText()
            self.lib.fjb_noise_destroy(self.handle, C.byref(err.buf))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def visual_grain(recipe: "DeviceRecipe", grain, density_cmy, noise: "DeviceNoise | None" = None, scratch=None,
                 stream=None):
    """Grain on three CUDA density planes (C, M, Y) in place."""
    torch = _torch()
    lib = load_library()
    h, w = density_cmy[0].shape
    need = int(lib.fjb_visual_grain_scratch_bytes(w, h))
    if scratch is None:
        scratch = torch.empty((need + 3) // 4, dtype=torch.float32, device=density_cmy[0].device)
    err = abi.ErrorText()
    st = lib.fjb_visual_grain(recipe.handle, C.byref(grain), noise.handle if noise is not None else None,
                              *[C.c_void_p(_ptr(t)) for t in density_cmy], density_cmy[0].stride(0), w, h,
                              C.c_void_p(_ptr(scratch)), scratch.numel() * 4, C.c_void_p(_stream_handle(stream)),
                              C.byref(err.buf))
    _check("fjb_visual_grain", st, err)


class Owner:
    """The drop-in boundary: fj_cuda_create / inspect / render / destroy over CUDA tensors."""

    def __init__(self):
        self.lib = load_library()
        self.handle = C.c_void_p()
        err = abi.ErrorText()
        _check("fj_cuda_create", self.lib.fj_cuda_create(C.byref(self.handle), C.byref(err.buf)), err)

    def close(self):
        if self.handle:
            err = abi.ErrorText()
            self.lib.fj_cuda_destroy(self.handle, C.byref(err.buf))
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_print_form(self, form: int):
        err = abi.ErrorText()
        _check("fjb_owner_set_print_form", self.lib.fjb_owner_set_print_form(self.handle, form, C.byref(err.buf)), err)

    def set_autotune(self, enable: bool):
        """Diffusion form autotuning (fjb_owner_set_autotune)."""
        err = abi.ErrorText()
        _check("fjb_owner_set_autotune", self.lib.fjb_owner_set_autotune(self.handle, 1 if enable else 0,
                                                                          C.byref(err.buf)), err)

    def diffusion_form(self, width: int, height: int, radius_px: int) -> int:
        """The owner's diffusion form decision (FJB_DIFFUSION_*, -1 undecided)."""
        err = abi.ErrorText()
        v = C.c_int32()
        _check("fjb_owner_diffusion_form", self.lib.fjb_owner_diffusion_form(self.handle, width, height, radius_px,
                                                                              C.byref(v), C.byref(err.buf)), err)
        return int(v.value)

    @staticmethod
    def _frame(src, dst, window=None, stream=None):
        h, w, comps = src.shape
        fr = abi.FjFrame()
        for im, t in ((fr.source, src), (fr.destination, dst)):
            im.address = _ptr(t)
            im.bounds = abi.FjRect(0, 0, w, h)
            im.row_bytes = t.stride(0) * 4
            im.components = comps
            im.depth = abi.FJ_DEPTH_FLOAT32
        fr.render_window = abi.FjRect(*(window or (0, 0, w, h)))
        fr.full_frame_extent = abi.FjRect(0, 0, w, h)
        if stream is not None:
            fr.stream = _stream_handle(stream)
            fr.flags |= abi.FJ_FRAME_STREAM_PRESENT
        return fr

    def render_batch(self, prepared, srcs, dsts, stream, graph_token: int = 0, frame_tokens=None):
        """fjb_render_batch over lists of records and (H, W, comps) float32 CUDA tensors,
        on `stream` (a torch.cuda.Stream). Returns the list of FjRenderOutcome (raises on
        a failed batch status); the diagnostic text is kept in `last_batch_text`."""
        n = len(prepared)
        frames = (abi.FjFrame * max(n, 1))()
        subs = (abi.FjSubmission * max(n, 1))()
        ptrs = (C.c_void_p * max(n, 1))()
        for i in range(n):
            frames[i] = self._frame(srcs[i], dsts[i])
            subs[i].frame_token = frame_tokens[i] if frame_tokens else 0
            ptrs[i] = C.cast(prepared[i].pointer(), C.c_void_p)
        err = abi.ErrorText()
        ctx = abi.FjCudaContext()
        if n:
            _check("fj_cuda_inspect", self.lib.fj_cuda_inspect(self.handle, C.byref(frames[0]), C.byref(ctx),
                                                               C.byref(err.buf)), err)
        outs = (abi.FjRenderOutcome * max(n, 1))()
        st = self.lib.fjb_render_batch(self.handle, C.byref(ctx), frames, subs, ptrs, n,
                                       C.c_void_p(_stream_handle(stream)), graph_token, outs, C.byref(err.buf))
        _check("fjb_render_batch", st, err)
        self.last_batch_text = err.text
        return [outs[i] for i in range(n)]

    def render(self, prepared, src, dst, window=None, stream=None, abort=None, frame_token: int = 0):
        """src/dst: (H, W, comps) float32 CUDA tensors covering the full frame; returns
        the FjRenderOutcome (raises on a failed status)."""
        fr = self._frame(src, dst, window, stream)
        err = abi.ErrorText()
        ctx = abi.FjCudaContext()
        _check("fj_cuda_inspect", self.lib.fj_cuda_inspect(self.handle, C.byref(fr), C.byref(ctx), C.byref(err.buf)), err)
        sub = abi.FjSubmission()
        sub.frame_token = frame_token
        query = abi.FjAbortQuery(abort or (lambda user: abi.FJ_ABORT_CONTINUE))
        cb = abi.FjAbortCallback(query, None)
        out = self.lib.fj_cuda_render(self.handle, C.byref(ctx), C.byref(fr), C.byref(sub), prepared.pointer(), cb,
                                      C.byref(err.buf))
        _check("fj_cuda_render", out.status, err)
        return out


def render_from_density_post(recipe: "DeviceRecipe", post, seed: int, origin, density_cmy, dst, src=None,
                             stream=None, scratch=None):
    """fjb_render_from_density_post on CUDA tensors: density planes (C, M, Y) -> print ->
    scan with scanner glare -> lens blur -> unsharp -> dst (H, W, comps)."""
    torch = _torch()
    lib = recipe.lib
    h, w = density_cmy[0].shape
    comps = dst.shape[2]
    need = int(lib.fjb_scanner_post_scratch_bytes(w, h))
    if scratch is None:
        scratch = torch.empty(need // 4, dtype=torch.float32, device=dst.device)
    err = abi.ErrorText()
    st = lib.fjb_render_from_density_post(
        recipe.handle, C.byref(post), seed, origin[0], origin[1], *[C.c_void_p(_ptr(t)) for t in density_cmy],
        C.c_void_p(_ptr(src) if src is not None else 0), (src.stride(0) * 4) if src is not None else 0,
        C.c_void_p(_ptr(dst)), dst.stride(0) * 4, w, h, comps, C.c_void_p(_ptr(scratch)), scratch.numel() * 4,
        C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_render_from_density_post", st, err)
    return scratch


def film_defects(effects: "abi.FjFilmEffects", density_cmy, dust=None, stream=None, table: bool = True):
    """fjb_film_defects on CUDA density planes (C, M, Y), in place: film scratches scale
    the densities; the film dust transmittance goes to `dust` (allocated when None and
    film dust is on). `table`: pass the particle-table scratch (False: the tiles build
    their candidates themselves). Returns the dust plane (or None)."""
    torch = _torch()
    lib = load_library()
    h, w = density_cmy[0].shape
    if dust is None and effects.film_dust.slot_probability > 0.0:
        dust = torch.empty((h, w), dtype=torch.float32, device=density_cmy[0].device)
    need = int(lib.fjb_film_defects_scratch_bytes(C.byref(effects), w, h)) if table else 0
    scratch = torch.empty(max(need, 4) // 4, dtype=torch.float32, device=density_cmy[0].device) if need else None
    err = abi.ErrorText()
    st = lib.fjb_film_defects(C.byref(effects), w, h, *[C.c_void_p(_ptr(t)) for t in density_cmy],
                              C.c_void_p(_ptr(dust) if dust is not None else 0),
                              C.c_void_p(_ptr(scratch) if scratch is not None else 0), need,
                              C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_film_defects", st, err)
    return dust


def gate_mask(effects: "abi.FjFilmEffects", stream=None, table: bool = True):
    """fjb_gate_mask: the gate transmittance grid (gate_height, gate_width) on the GPU."""
    torch = _torch()
    lib = load_library()
    mask = torch.empty((max(effects.gate_height, 1), max(effects.gate_width, 1)), dtype=torch.float32, device="cuda")
    need = int(lib.fjb_gate_mask_scratch_bytes(C.byref(effects), effects.gate_width, effects.gate_height)) if table else 0
    scratch = torch.empty(max(need, 4) // 4, dtype=torch.float32, device="cuda") if need else None
    err = abi.ErrorText()
    st = lib.fjb_gate_mask(C.byref(effects), C.c_void_p(_ptr(mask)), effects.gate_width, effects.gate_height,
                           C.c_void_p(_ptr(scratch) if scratch is not None else 0), need,
                           C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_gate_mask", st, err)
    return mask


def render_from_density_effects(recipe: "DeviceRecipe", post, seed: int, origin, effects, dust, mask, density_cmy,
                                dst, src=None, stream=None, scratch=None):
    """fjb_render_from_density_effects: render_from_density_post with the film dust plane
    and, with the gate output on, weave and the gate mask at the encoding."""
    torch = _torch()
    lib = recipe.lib
    h, w = density_cmy[0].shape
    comps = dst.shape[2]
    need = int(lib.fjb_scanner_post_scratch_bytes(w, h))
    if scratch is None:
        scratch = torch.empty(need // 4, dtype=torch.float32, device=dst.device)
    err = abi.ErrorText()
    st = lib.fjb_render_from_density_effects(
        recipe.handle, C.byref(post), seed, origin[0], origin[1], C.byref(effects) if effects is not None else None,
        C.c_void_p(_ptr(dust) if dust is not None else 0), C.c_void_p(_ptr(mask) if mask is not None else 0),
        *[C.c_void_p(_ptr(t)) for t in density_cmy],
        C.c_void_p(_ptr(src) if src is not None else 0), (src.stride(0) * 4) if src is not None else 0,
        C.c_void_p(_ptr(dst)), dst.stride(0) * 4, w, h, comps, C.c_void_p(_ptr(scratch)), scratch.numel() * 4,
        C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_render_from_density_effects", st, err)
    return scratch


def tc_lut_build(spectra, sensitivity_rgb, reference_illuminant, white_xyz, method: int = 0,
                 spectral_blur: float = 0.0, surface=None, compression: bool = False, hull=None, stream=None):
    """fjb_tc_lut_build: the film TC LUT (192 * 192 * 4 floats on the GPU) from CUDA
    spectra (192 * 192 * 81 floats) and host sensitivity (81 x 3) / illuminant (81)."""
    import numpy as np

    torch = _torch()
    lib = load_library()
    sens = np.ascontiguousarray(sensitivity_rgb, np.float32).reshape(-1)
    ill = np.ascontiguousarray(reference_illuminant, np.float32).reshape(-1)
    table = torch.empty(192 * 192 * 4, dtype=torch.float32, device=spectra.device)
    inp = abi.FjbTcLutInput()
    inp.spectra = _ptr(spectra)
    inp.sensitivity_rgb = sens.ctypes.data_as(C.POINTER(C.c_float))
    inp.reference_illuminant = ill.ctypes.data_as(C.POINTER(C.c_float))
    for i in range(3):
        inp.projection_white_xyz[i] = float(white_xyz[i])
    inp.spectral_blur = spectral_blur
    inp.method = method
    if surface is not None:
        surf = np.ascontiguousarray(surface, np.float32).reshape(-1)
        inp.apply_surface = 1
        inp.surface_rgb = surf.ctypes.data_as(C.POINTER(C.c_float))
    if compression:
        inp.input_compression = 1
        if hull is not None:
            xy = np.ascontiguousarray(hull[1], np.float32).reshape(-1)
            inp.hull_xy = xy.ctypes.data_as(C.POINTER(C.c_float))
            inp.hull_center[0], inp.hull_center[1] = float(hull[0][0]), float(hull[0][1])
            inp.hull_available = 1
    err = abi.ErrorText()
    st = lib.fjb_tc_lut_build(C.byref(inp), C.c_void_p(_ptr(table)), C.c_void_p(_stream_handle(stream)),
                              C.byref(err.buf))
    _check("fjb_tc_lut_build", st, err)
    return table


def highlight_boost(descriptor: "abi.FjHighlightBoost", carrier_bgr, stream=None, state=None):
    """In-place highlight reconstruction on CUDA carrier planes (B, G, R), then the
    disposition check (raises FjError on an invalid carrier or a peak overflow). Returns
    the disposition (0 bypass, 1 applied)."""
    torch = _torch()
    lib = load_library()
    b, g, r = carrier_bgr
    h, w = b.shape
    if state is None:
        state = torch.zeros(int(lib.fjb_highlight_boost_state_bytes()) // 4, dtype=torch.int32, device=b.device)
    err = abi.ErrorText()
    st = lib.fjb_highlight_boost(C.byref(descriptor), C.c_void_p(_ptr(b)), C.c_void_p(_ptr(g)), C.c_void_p(_ptr(r)),
                                 b.stride(0), w, h, C.c_void_p(_ptr(state)), C.c_void_p(_stream_handle(stream)),
                                 C.byref(err.buf))
    _check("fjb_highlight_boost", st, err)
    disp = C.c_uint32()
    st = lib.fjb_highlight_boost_result(C.c_void_p(_ptr(state)), C.c_void_p(_stream_handle(stream)), C.byref(disp),
                                        C.byref(err.buf))
    _check("fjb_highlight_boost_result", st, err)
    return disp.value
