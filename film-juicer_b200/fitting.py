"""Fitting recipe parameters to target renders: a torch.autograd.Function over the
library's fitting entry points (fjb_fit_forward, fjb_fit_vjp) and an Adam loop on it.

The differentiable function is the per-pixel chain of a recipe (camera exposure, film
curves, negative-donor DIR with its compensated axes, print exposure and curves on the
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
