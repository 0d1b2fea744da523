"""Fitting recipe parameters to target renders: a torch.autograd.Function over the
library's fitting entry points (fjb_fit_forward, fjb_fit_vjp) and an Adam loop on it.

The differentiable function is the per-pixel chain of a recipe (camera exposure, film
curves, DIR couplers (negative-donor with its compensated axes, or the positive stocks'
receiver Langmuir), print exposure and curves on the
print route, scanner LUT, correction and colour matrices) from a source image to the
scanner's linear output RGB, as a function of 13 parameters (FjbFitParams order):

    0-2   exposure_ev B, G, R   film exposure times 2^ev
    3-5   film_gamma B, G, R    gamma factor of the film and compensated curves
    6-8   print_gamma C, M, Y   gamma factor of the print curves (1 = the recipe's)
    9-11  donor_k B, G, R       DIR donor Langmuir knees (absolute, as FjDirCouplers)
    12    print_ev              print exposure times 2^ev

The backward pass is the library's hand-written adjoint: it recomputes each pixel's
forward values (the print's 81 spectral transmittances included) and sums the pixels'
vector-Jacobian products in FP64 in a fixed order. A batch of crops that share the
parameters is one tall image (crops stacked along rows): the chain is per pixel.

torch provides device memory and autograd plumbing; every pixel and every gradient is
computed by the CUDA library. Without the library or a GPU this module raises.
"""
from __future__ import annotations

import ctypes as C

from . import abi, load_library
from .runtime import DeviceRecipe, _check, _ptr, _stream_handle, _torch

PARAM_NAMES = tuple(abi.FJB_FIT_PARAM_NAMES)
N_PARAMS = len(PARAM_NAMES)


def _params(theta) -> abi.FjbFitParams:
    v = [float(x) for x in theta.detach().to("cpu", dtype=theta.dtype).tolist()]
    if len(v) != N_PARAMS:
        raise ValueError(f"theta must hold {N_PARAMS} parameters, got {len(v)}")
    p = abi.FjbFitParams()
    for i in range(3):
        p.exposure_ev[i] = v[i]
        p.film_gamma[i] = v[3 + i]
        p.print_gamma[i] = v[6 + i]
        p.donor_k[i] = v[9 + i]
    p.print_ev = v[12]
    return p


def default_theta(recipe: DeviceRecipe, dtype=None):
    """The parameters that reproduce the recipe (fjb_fit_defaults), a float64 CPU tensor."""
    torch = _torch()
    p = abi.FjbFitParams()
    err = abi.ErrorText()
    _check("fjb_fit_defaults", recipe.lib.fjb_fit_defaults(recipe.handle, C.byref(p), C.byref(err.buf)), err)
    vals = list(p.exposure_ev) + list(p.film_gamma) + list(p.print_gamma) + list(p.donor_k) + [p.print_ev]
    return torch.tensor(vals, dtype=dtype or torch.float64)


def forward(recipe: DeviceRecipe, theta, src, out=None, stream=None):
    """Linear output RGB planes (3, H, W) float32 of src (H, W, 3|4) float32 CUDA for theta."""
    torch = _torch()
    h, w, comps = src.shape
    if out is None:
        out = torch.empty((3, h, w), dtype=torch.float32, device=src.device)
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_forward(recipe.handle, C.byref(params), C.c_void_p(_ptr(src)), src.stride(0) * 4, comps,
                                    *[C.c_void_p(_ptr(out[c])) for c in range(3)], w, h,
                                    C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_fit_forward", st, err)
    return out


class _Scratch:
    def __init__(self):
        self.buf = None

    def get(self, torch, device):
        nbytes = int(load_library().fjb_fit_scratch_bytes())
        if self.buf is None or self.buf.numel() < nbytes or self.buf.device != device:
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        return self.buf


_SCRATCH = _Scratch()


def vjp(recipe: DeviceRecipe, theta, src, grad_rgb, grad_out=None, stream=None):
    """sum over pixels of grad_rgb^T d rgb / d theta, a (13,) float64 CUDA tensor.
    grad_rgb: (3, H, W) float32 CUDA planes (contiguous)."""
    torch = _torch()
    h, w, comps = src.shape
    g = grad_rgb.contiguous().to(torch.float32)
    if grad_out is None:
        grad_out = torch.empty(N_PARAMS, dtype=torch.float64, device=src.device)
    scratch = _SCRATCH.get(torch, src.device)
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_vjp(recipe.handle, C.byref(params), C.c_void_p(_ptr(src)), src.stride(0) * 4, comps,
                                *[C.c_void_p(_ptr(g[c])) for c in range(3)], w, h, C.c_void_p(_ptr(grad_out)),
                                C.c_void_p(_ptr(scratch)), scratch.numel(), C.c_void_p(_stream_handle(stream)),
                                C.byref(err.buf))
    _check("fjb_fit_vjp", st, err)
    return grad_out


def _function():
    torch = _torch()

    class FitChain(torch.autograd.Function):
        """rgb = chain(theta; recipe, src); backward through fjb_fit_vjp."""

        @staticmethod
        def forward(ctx, theta, recipe, src):
            ctx.recipe = recipe
            ctx.save_for_backward(theta, src)
            return forward(recipe, theta, src)

        @staticmethod
        def backward(ctx, grad_rgb):
            theta, src = ctx.saved_tensors
            g = vjp(ctx.recipe, theta, src, grad_rgb)
            return g.to(device=theta.device, dtype=theta.dtype), None, None

    return FitChain


_FN = None


def chain(theta, recipe: DeviceRecipe, src):
    """Differentiable linear output RGB (3, H, W) of src for theta (13,)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(theta, recipe, src)


def stack_crops(crops):
    """A batch of crops (B, H, W, C) as one (B*H, W, C) image (the chain is per pixel)."""
    b, h, w, c = crops.shape
    return crops.reshape(b * h, w, c)


def fit(recipe: DeviceRecipe, src, target, theta0, *, free=None, steps: int = 200, lr: float = 0.02,
        callback=None):
    """Fits theta to a target linear render by Adam on the mean squared error.

    src: (H, W, 3|4) float32 CUDA source (a crop batch via stack_crops); target: (3, H, W)
    linear output RGB; theta0: (13,) starting parameters; free: indices of the parameters
    to fit (default: all). Pixels that the chain rejects (NaN) in the target or the
    render are left out of the loss. Returns (theta, losses)."""
    torch = _torch()
    theta0 = theta0.detach().to(torch.float64).cpu()
    free = list(range(N_PARAMS)) if free is None else list(free)
    mask = torch.zeros(N_PARAMS, dtype=torch.float64)
    mask[free] = 1.0
    var = theta0[free].clone().requires_grad_(True)
    opt = torch.optim.Adam([var], lr=lr)
    valid_t = torch.isfinite(target)
    losses = []
    for step in range(steps):
        opt.zero_grad()
        theta = theta0 * (1.0 - mask)
        theta = theta.index_put((torch.tensor(free),), var)
        rgb = chain(theta, recipe, src)
        valid = valid_t & torch.isfinite(rgb.detach())
        diff = torch.where(valid, rgb - target, torch.zeros_like(rgb))
        loss = (diff * diff).sum() / valid.sum().clamp(min=1)
        loss.backward()
        opt.step()
        with torch.no_grad():  # donor knees stay positive
            for j, i in enumerate(free):
                if 9 <= i <= 11:
                    var[j].clamp_(min=1e-3)
        losses.append(float(loss.detach()))
        if callback is not None:
            callback(step, theta.detach(), losses[-1])
    theta = theta0.clone()
    theta[free] = var.detach()
    return theta, losses


# ---------------------------------------------------------------------------
# Whole frames with the optics on: camera diffusion (scatter fraction f) and emulsion
# scatter (amount a) / halation back-reflection (strength s per channel) ahead of the
# per-pixel chain. Both stages are linear in the carrier and act per channel, so the
# exposure parameters (a per-channel scale) commute with them: the per-pixel chain runs
# from the post-optics carrier (fjb_fit_*_carrier) with exact gradients, and each
# optics parameter's gradient is <d L / d carrier, d carrier / d parameter>, the tangent
# plane obtained by running the same linear stages forward on it:
#   diffusion  x1 = (1 - f) x0 + f PSF*x0                 d x1 / d f = PSF*x0 - x0
#   scatter    x2 = (1 - a) x1 + a S(x1)                  d x2 / d a = S(x1) - x1
#   bounce     x3 = (x2 + s B(x2)) / (1 + s)  [renorm]    d x3 / d s = (B(x2) - x2) / (1 + s)^2
#                   x2 + s B(x2)              [else]                  = B(x2)
# with the tangents of f and a carried through the later stages (all linear).
# ---------------------------------------------------------------------------
OPTIC_NAMES = ("camera_scatter_fraction", "scatter_amount", "halation_strength_r", "halation_strength_g",
               "halation_strength_b")


def _copy(struct):
    return type(struct).from_buffer_copy(struct)


class FrameFit:
    """A frame's fitting problem: the recipe, the frame's optics descriptors and its
    camera exposure (computed once by the library: the optics parameters act after it).

    host: the frame's FjPreparedHostData (a HostRecord's `.h`), with camera diffusion,
    scatter/halation, spatial DIR, auto exposure and highlight reconstruction switched
    by its records (the metered scale and the reconstructed highlights are taken once
    from the source: they do not depend on the parameters); grain and enlarger
    diffusion are outside this chain and must be off. src: (H, W, 3|4) float32 CUDA
    source.

    With spatial DIR the development subtracts the filtered donor corrections: the
    forward is the source stage, the frame's DIR filter and the development; the
    adjoint runs the development's adjoint (theta, carrier and filtered-correction
    gradients), filters the correction cotangent with the same filter (it is
    symmetric, its own adjoint) and adds the source stage's adjoint."""

    def __init__(self, recipe: DeviceRecipe, host, src, stream=None):
        torch = _torch()
        o = host.optics
        if (host.grain.flags & abi.FJ_GRAIN_ACTIVE) or (o.flags & abi.FJ_OPTICS_ENLARGER_DIFFUSION):
            raise ValueError("frame fitting covers camera diffusion, scatter/halation, spatial DIR, auto exposure "
                             "and highlight reconstruction")
        self.spatial = _copy(host.spatial_dir) if host.spatial_dir.component_count else None
        self._dir_filter = None
        self.recipe, self.stream = recipe, stream
        self.diffusion_on = bool(o.flags & abi.FJ_OPTICS_CAMERA_DIFFUSION)
        self.halation_on = bool(o.flags & abi.FJ_OPTICS_SCATTER_HALATION)
        self.camera = _copy(o.camera)
        self.halation = _copy(o.scatter_halation)
        if self.diffusion_on:
            from .runtime import diffusion_components

            self.components = diffusion_components(self.camera)
        h, w = src.shape[0], src.shape[1]
        self.shape = (h, w)
        planes = [torch.empty((h, w), dtype=torch.float32, device=src.device) for _ in range(3)]
        self.meter_scale = None
        if host.film_exposure.flags & abi.FJ_FILM_AUTO_EXPOSURE:
            # the metered scale is a function of the source alone: metered once, it sits
            # in the carrier, and the parameters act after it as they do without metering
            from .runtime import auto_exposure

            self.meter_scale = torch.empty(1, dtype=torch.float32, device=src.device)
            auto_exposure(recipe, src, host.auto_exposure, self.meter_scale, stream=stream)
            recipe.set_exposure_scale_device(self.meter_scale)
        try:
            recipe.camera_exposure(src, planes, stream=stream)  # B, G, R
        finally:
            if self.meter_scale is not None:
                recipe.set_exposure_scale_device(None)
        if o.flags & abi.FJ_OPTICS_HIGHLIGHT_BOOST:
            # highlight reconstruction acts on the camera exposure before the optics and
            # depends on the source alone: applied once, it is part of the carrier
            from .runtime import highlight_boost

            highlight_boost(o.highlight_boost, planes, stream=stream)
        self.x0 = [planes[2], planes[1], planes[0]]  # R, G, B
        self._scratch = None

    def optics_default(self):
        """The frame's own optics parameters (OPTIC_NAMES order), float64 CPU."""
        torch = _torch()
        ch = self.halation.channels
        return torch.tensor([self.camera.scatter_fraction, self.halation.scatter_amount, ch[0].total_strength,
                             ch[1].total_strength, ch[2].total_strength], dtype=torch.float64)

    # -- the linear optics stages, on three R, G, B planes --
    def _diffuse(self, planes, fraction):
        from .runtime import diffusion

        torch = _torch()
        out = [torch.empty_like(p) for p in planes]
        diffusion(self.components, int(self.camera.radius_px), float(fraction), planes, out, stream=self.stream)
        return out

    def _halation(self, planes, amount, strengths, renormalize=None):
        """In place: scatter with `amount`, then back-reflection with `strengths`."""
        from .runtime import scatter_halation

        d = _copy(self.halation)
        d.scatter_amount = float(amount)
        for c in range(3):
            d.channels[c].total_strength = float(strengths[c])
        if renormalize is not None:
            d.renormalize = 1 if renormalize else 0
        if d.scatter_amount == 0.0 and all(float(s) == 0.0 for s in strengths):
            return planes
        self._scratch = scatter_halation(d, planes, stream=self.stream, scratch=self._scratch)
        return planes

    def carriers(self, optics):
        """(x1, x2, x3): after diffusion, after scatter, after back-reflection (R, G, B)."""
        v = [float(x) for x in optics.detach().cpu().tolist()]
        x1 = self._diffuse(self.x0, v[0]) if self.diffusion_on else [p.clone() for p in self.x0]
        x2 = [p.clone() for p in x1]
        x3 = [p.clone() for p in x1]
        if self.halation_on:
            self._halation(x2, v[1], (0.0, 0.0, 0.0))
            x3 = [p.clone() for p in x2]
            self._halation(x3, 0.0, v[2:5])
        return x1, x2, x3

    def tangents(self, optics, x1, x2):
        """d carrier / d optics parameter, five lists of R, G, B planes (None where the
        frame's stage is off, or for the halation strength of a channel the frame's
        record gives no back-reflection: the carrier does not depend on it)."""
        v = [float(x) for x in optics.detach().cpu().tolist()]
        out = [None] * 5
        if self.diffusion_on:
            t = [a - b for a, b in zip(self._diffuse(self.x0, 1.0), self.x0)]
            if self.halation_on:
                self._halation(t, v[1], (0.0, 0.0, 0.0))
                self._halation(t, 0.0, v[2:5])
            out[0] = t
        if self.halation_on:
            s1 = self._halation([p.clone() for p in x1], 1.0, (0.0, 0.0, 0.0))
            t = [a - b for a, b in zip(s1, x1)]
            self._halation(t, 0.0, v[2:5])
            out[1] = t
            renorm = bool(self.halation.renormalize)
            b1 = self._halation([p.clone() for p in x2], 0.0, (1.0, 1.0, 1.0), renormalize=False)
            torch = _torch()
            for c in range(3):
                if self.halation.channels[c].total_strength == 0.0:
                    # no back-reflection configured for this channel (its Gaussians are
                    # not part of the record): not a free parameter
                    continue
                t = [torch.zeros_like(p) for p in x2]
                bc = b1[c] - x2[c]  # B(x2) of channel c
                t[c] = (bc - x2[c]) / (1.0 + v[2 + c]) ** 2 if renorm else bc
                out[2 + c] = t
        return out

    def dir_filter(self, planes_ymc):
        """The frame's spatial DIR filter of three (H, W) planes (Y, M, C), prepared once
        per frame (runtime.DirFilter)."""
        from .runtime import DirFilter

        torch = _torch()
        if self._dir_filter is None:
            h, w = self.shape
            self._dir_filter = DirFilter(self.spatial, w, h, stream=self.stream)
        out = [torch.empty_like(p) for p in planes_ymc]
        return self._dir_filter.apply([p.contiguous() for p in planes_ymc], out, stream=self.stream)

    def close(self):
        """Frees the prepared DIR filter (also done when the object is collected)."""
        if self._dir_filter is not None:
            self._dir_filter.close()
            self._dir_filter = None

    def filtered_corrections(self, theta, carrier_rgb):
        """Spatial DIR: the filtered donor corrections (Y, M, C) for theta."""
        return self.dir_filter(dir_source_carrier(self.recipe, theta, carrier_rgb, stream=self.stream))

    def forward(self, theta, optics, out=None):
        """Linear output RGB planes (3, H, W) of the frame for theta (13) and optics (5)."""
        _, _, x3 = self.carriers(optics)
        if self.spatial is not None:
            cf = self.filtered_corrections(theta, x3)
            return forward_spatial_carrier(self.recipe, theta, x3, cf, out=out, stream=self.stream)
        return forward_carrier(self.recipe, theta, x3, out=out, stream=self.stream)

    def vjp_carrier(self, theta, carrier_rgb, grad_rgb):
        """(d L / d theta (13,) float64 CUDA, d L / d carrier (R, G, B planes)) of the
        chain after the optics, spatial DIR included."""
        if self.spatial is None:
            return vjp_carrier(self.recipe, theta, carrier_rgb, grad_rgb, stream=self.stream)
        cf = self.filtered_corrections(theta, carrier_rgb)
        g_dev, g_carrier, g_cf = vjp_spatial_carrier(self.recipe, theta, carrier_rgb, cf, grad_rgb,
                                                     stream=self.stream)
        g_src = self.dir_filter(g_cf)
        g_source = dir_source_vjp_carrier(self.recipe, theta, carrier_rgb, g_src, grad_carrier_rgb=g_carrier,
                                          stream=self.stream)
        return g_dev + g_source, g_carrier

    def vjp(self, theta, optics, grad_rgb):
        """(d L / d theta (13,), d L / d optics (5,)) for L = <grad_rgb, rgb>, float64 CPU."""
        torch = _torch()
        x1, x2, x3 = self.carriers(optics)
        g_theta, g_carrier = self.vjp_carrier(theta, x3, grad_rgb)
        g_opt = torch.zeros(len(OPTIC_NAMES), dtype=torch.float64)
        for i, t in enumerate(self.tangents(optics, x1, x2)):
            if t is not None:
                g_opt[i] = sum(float((g.double() * p.double()).sum()) for g, p in zip(g_carrier, t))
        return g_theta.cpu(), g_opt


def forward_carrier(recipe: DeviceRecipe, theta, carrier_rgb, out=None, stream=None):
    """fjb_fit_forward_carrier on carrier planes (R, G, B lists of (H, W) CUDA tensors)."""
    torch = _torch()
    r, g, b = carrier_rgb
    h, w = r.shape
    if out is None:
        out = torch.empty((3, h, w), dtype=torch.float32, device=r.device)
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_forward_carrier(recipe.handle, C.byref(params), *[C.c_void_p(_ptr(t)) for t in (b, g, r)],
                                            r.stride(0), *[C.c_void_p(_ptr(out[c])) for c in range(3)], w, h,
                                            C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_fit_forward_carrier", st, err)
    return out


def vjp_carrier(recipe: DeviceRecipe, theta, carrier_rgb, grad_rgb, stream=None):
    """fjb_fit_vjp_carrier: (d L / d theta (13,) float64 CUDA, d L / d carrier as R, G, B
    planes) for L = <grad_rgb, rgb>."""
    torch = _torch()
    r, g, b = carrier_rgb
    h, w = r.shape
    gr = grad_rgb.contiguous().to(torch.float32)
    grad = torch.empty(N_PARAMS, dtype=torch.float64, device=r.device)
    gc = [torch.empty((h, w), dtype=torch.float32, device=r.device) for _ in range(3)]  # B, G, R
    scratch = _SCRATCH.get(torch, r.device)
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_vjp_carrier(recipe.handle, C.byref(params), *[C.c_void_p(_ptr(t)) for t in (b, g, r)],
                                        r.stride(0), *[C.c_void_p(_ptr(gr[c])) for c in range(3)], w, h,
                                        C.c_void_p(_ptr(grad)), *[C.c_void_p(_ptr(t)) for t in gc],
                                        C.c_void_p(_ptr(scratch)), scratch.numel(),
                                        C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_fit_vjp_carrier", st, err)
    return grad, [gc[2], gc[1], gc[0]]


def _planes(ts):
    return [C.c_void_p(_ptr(t)) for t in ts]


def dir_source_carrier(recipe: DeviceRecipe, theta, carrier_rgb, stream=None):
    """fjb_fit_dir_source_carrier: the donor corrections for theta as (Y, M, C) planes
    (the B, G, R receivers), before the spatial DIR filter."""
    torch = _torch()
    r, g, b = carrier_rgb
    h, w = r.shape
    out = [torch.empty((h, w), dtype=torch.float32, device=r.device) for _ in range(3)]
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_dir_source_carrier(recipe.handle, C.byref(params), *_planes((b, g, r)), r.stride(0),
                                               *_planes(out), w, h, C.c_void_p(_stream_handle(stream)),
                                               C.byref(err.buf))
    _check("fjb_fit_dir_source_carrier", st, err)
    return out


def forward_spatial_carrier(recipe: DeviceRecipe, theta, carrier_rgb, filtered_ymc, out=None, stream=None):
    """fjb_fit_forward_spatial_carrier: linear output RGB (3, H, W) developed with the
    filtered DIR corrections (Y, M, C planes)."""
    torch = _torch()
    r, g, b = carrier_rgb
    h, w = r.shape
    if out is None:
        out = torch.empty((3, h, w), dtype=torch.float32, device=r.device)
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_forward_spatial_carrier(recipe.handle, C.byref(params), *_planes((b, g, r)), r.stride(0),
                                                    *_planes(filtered_ymc), *_planes([out[c] for c in range(3)]), w, h,
                                                    C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_fit_forward_spatial_carrier", st, err)
    return out


def vjp_spatial_carrier(recipe: DeviceRecipe, theta, carrier_rgb, filtered_ymc, grad_rgb, stream=None):
    """fjb_fit_vjp_spatial_carrier: (d L / d theta of the development (13,) float64
    CUDA, d L / d carrier (R, G, B planes), d L / d filtered corrections (Y, M, C))."""
    torch = _torch()
    r, g, b = carrier_rgb
    h, w = r.shape
    gr = grad_rgb.contiguous().to(torch.float32)
    grad = torch.empty(N_PARAMS, dtype=torch.float64, device=r.device)
    gc = [torch.empty((h, w), dtype=torch.float32, device=r.device) for _ in range(3)]  # B, G, R
    gf = [torch.empty((h, w), dtype=torch.float32, device=r.device) for _ in range(3)]  # Y, M, C
    scratch = _SCRATCH.get(torch, r.device)
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_vjp_spatial_carrier(recipe.handle, C.byref(params), *_planes((b, g, r)), r.stride(0),
                                                *_planes(filtered_ymc), *_planes([gr[c] for c in range(3)]), w, h,
                                                C.c_void_p(_ptr(grad)), *_planes(gc), *_planes(gf),
                                                C.c_void_p(_ptr(scratch)), scratch.numel(),
                                                C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_fit_vjp_spatial_carrier", st, err)
    return grad, [gc[2], gc[1], gc[0]], gf


def dir_source_vjp_carrier(recipe: DeviceRecipe, theta, carrier_rgb, grad_corr_ymc, grad_carrier_rgb=None,
                           stream=None):
    """fjb_fit_dir_source_vjp_carrier: d L / d theta (13,) float64 CUDA of the source
    stage for the corrections' cotangent; adds d L / d carrier into grad_carrier_rgb
    (R, G, B planes) when given."""
    torch = _torch()
    r, g, b = carrier_rgb
    h, w = r.shape
    grad = torch.empty(N_PARAMS, dtype=torch.float64, device=r.device)
    scratch = _SCRATCH.get(torch, r.device)
    gc = [C.c_void_p(0)] * 3 if grad_carrier_rgb is None else _planes(grad_carrier_rgb[::-1])  # B, G, R
    params = _params(theta)
    err = abi.ErrorText()
    st = recipe.lib.fjb_fit_dir_source_vjp_carrier(recipe.handle, C.byref(params), *_planes((b, g, r)), r.stride(0),
                                                   *_planes(grad_corr_ymc), w, h, C.c_void_p(_ptr(grad)), *gc,
                                                   C.c_void_p(_ptr(scratch)), scratch.numel(),
                                                   C.c_void_p(_stream_handle(stream)), C.byref(err.buf))
    _check("fjb_fit_dir_source_vjp_carrier", st, err)
    return grad


def _frame_function():
    torch = _torch()

    class FrameChain(torch.autograd.Function):
        """rgb = chain(theta, optics; frame); backward: the carrier adjoint and the
        optics tangents."""

        @staticmethod
        def forward(ctx, theta, optics, frame):
            ctx.frame = frame
            ctx.save_for_backward(theta, optics)
            return frame.forward(theta, optics)

        @staticmethod
        def backward(ctx, grad_rgb):
            theta, optics = ctx.saved_tensors
            g_theta, g_opt = ctx.frame.vjp(theta, optics, grad_rgb)
            return (g_theta.to(device=theta.device, dtype=theta.dtype),
                    g_opt.to(device=optics.device, dtype=optics.dtype), None)

    return FrameChain


_FRAME_FN = None


def frame_chain(theta, optics, frame: FrameFit):
    """Differentiable linear output RGB (3, H, W) of a frame with its optics on."""
    global _FRAME_FN
    if _FRAME_FN is None:
        _FRAME_FN = _frame_function()
    return _FRAME_FN.apply(theta, optics, frame)
