"""FP64 PyTorch transcription of the per-pixel chain as a function of the fitting
parameters (TEST ORACLE).

Test infrastructure: only tests/ load it, as the checker of the library's fitting
entry points (fjb_fit_forward, fjb_fit_vjp); the product never imports it.

The chain is the capture-to-scan chain of the render (src/Cuda/JuicerCudaDeviceHelpers.cuh:
563-1071, src/Cuda/Scan/JuicerCudaScanPipeline.cu:1700-1811) restated in FP64 with
autograd, on the tables the oracle packs from the same FjPreparedHostData
(oracle.c oracle_fit_tables, oracle_scanner_lut): the camera exposure of each pixel (the
oracle's FP32 film exposure with the route correction) times 2^ev, log10, the film
curves at logE * gamma, the DIR couplers (negative stocks: Langmuir donors, the coupler
matrix and the compensated curves, whose axes are rebuilt from the donor knees as the
reference's host builds them: rust/film-juicer-core/src/film/dir.rs:258-290; positive
stocks: donors dmax - density, the coupler matrix and the receivers' Langmuir, on the
recipe's axes), on the print route
the spectral print exposure 10^-(D . eps + base) x illuminant x sensitivity with the
mid-grey normaliser, preflash, print exposure x 2^print_ev and route correction, log10
and the print curves at logP * print_gamma, then the scanner's PCHIP LUT (the reference's
Hermite evaluation order, cell clamp), exp2, the scanner correction and the CAT02 /
output matrices. Output: the linear output RGB (before gamut compression and encoding).

Parameters theta (13, FjbFitParams order): exposure_ev B, G, R; film_gamma B, G, R;
print_gamma C, M, Y; donor_k B, G, R (absolute knees, as FjDirCouplers.donor_k_rgb);
print_ev.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as _orc

NL = 81
MAX_SAMPLES = 1024


class OracleFitTables(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("dir_mode", C.c_int32), ("print", C.c_int32), ("np", C.c_int32),
        ("medium_negative", C.c_int32), ("res", C.c_int32), ("corr_active", C.c_int32), ("pad", C.c_int32),
        ("log_exposure", C.c_float * MAX_SAMPLES),
        ("density_bgr", (C.c_float * MAX_SAMPLES) * 3),
        ("axes_bgr", (C.c_float * MAX_SAMPLES) * 3),
        ("gamma_bgr", C.c_float * 3), ("dir_m", C.c_float * 9), ("dir_dref", C.c_float * 3), ("dir_k", C.c_float * 3),
        ("eps_cmy", C.c_float * (NL * 3)), ("base", C.c_float * NL), ("illuminant", C.c_float * NL),
        ("sens_cmy", C.c_float * (NL * 3)),
        ("midgray", C.c_float), ("preflash", C.c_float), ("preflash_raw", C.c_float * 3),
        ("print_exposure", C.c_float), ("print_route", C.c_float),
        ("print_log_exposure", C.c_float * MAX_SAMPLES),
        ("print_density_cmy", (C.c_float * MAX_SAMPLES) * 3),
        ("min_cmy", C.c_float * 3), ("inv_cmy", C.c_float * 3), ("corr_slope", C.c_float), ("corr_offset", C.c_float),
        ("cat02", C.c_float * 9), ("xyz_to_rgb", C.c_float * 9),
        ("dir_dmax", C.c_float * 3), ("dir_rcref", C.c_float * 3), ("dir_rkr", C.c_float * 3),
    ]


def tables(record) -> dict:
    """The packed tables of `record` (a HostRecord) as float64 numpy arrays."""
    lib = _orc.load()
    fn = lib.oracle_fit_tables
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.POINTER(OracleFitTables)]
    t = OracleFitTables()
    rc = fn(record.pointer(), C.byref(t))
    if rc != 0:
        raise RuntimeError(f"oracle_fit_tables failed with code {rc}")
    n, npr = t.n, t.np
    f = lambda a, k=None: np.array(a[:k] if k is not None else a[:], dtype=np.float64)  # noqa: E731
    out = {
        "n": n, "dir_mode": t.dir_mode, "print": bool(t.print), "medium_negative": bool(t.medium_negative),
        "res": t.res, "corr_active": bool(t.corr_active),
        "log_exposure": f(t.log_exposure, n),
        "density_bgr": np.stack([f(t.density_bgr[c], n) for c in range(3)]),
        "axes_bgr": np.stack([f(t.axes_bgr[c], n) for c in range(3)]),
        "gamma_bgr": f(t.gamma_bgr), "dir_m": f(t.dir_m), "dir_dref": f(t.dir_dref), "dir_k": f(t.dir_k),
        "min_cmy": f(t.min_cmy), "inv_cmy": f(t.inv_cmy), "corr_slope": float(t.corr_slope),
        "corr_offset": float(t.corr_offset), "cat02": f(t.cat02), "xyz_to_rgb": f(t.xyz_to_rgb),
        "dir_dmax": f(t.dir_dmax), "dir_rcref": f(t.dir_rcref), "dir_rkr": f(t.dir_rkr),
    }
    if t.print:
        eps, base, ill = f(t.eps_cmy).reshape(NL, 3), f(t.base), f(t.illuminant)
        sens = f(t.sens_cmy).reshape(NL, 3)
        # A wavelength whose transmittance is NaN for every density (a NaN dye or base
        # density, a NaN illuminant) contributes nothing, as the reference's print
        # integral drops NaN transmittances (src/Cuda/JuicerCudaDeviceHelpers.cuh:860-864).
        dead = np.isnan(eps).any(axis=1) | np.isnan(base) | np.isnan(ill)
        eps[dead], base[dead], ill[dead], sens[dead] = 0.0, 0.0, 0.0, 0.0
        out.update({
            "eps_cmy": eps, "base": base, "illuminant": ill,
            "sens_cmy": sens, "midgray": float(t.midgray), "preflash": float(t.preflash),
            "preflash_raw": f(t.preflash_raw), "print_exposure": float(t.print_exposure),
            "print_route": float(t.print_route), "print_log_exposure": f(t.print_log_exposure, npr),
            "print_density_cmy": np.stack([f(t.print_density_cmy[c], npr) for c in range(3)]),
        })
    return out


def default_theta(tab: dict) -> np.ndarray:
    """The parameters that reproduce the recipe (fjb_fit_defaults)."""
    k = tab["dir_k"] if tab["dir_mode"] == 1 else np.ones(3)
    return np.concatenate([np.zeros(3), tab["gamma_bgr"], np.ones(3), k, [0.0]])


def perturbed_theta(tab: dict) -> np.ndarray:
    """A parameter point away from the recipe's own values (the gradient checks' point
    and the fitting tests' truth): exposure +0.2/-0.1/+0.15 ev, film gammas +0.05/-0.04/
    +0.03, print gammas +0.05/-0.06/+0.04, donor knees x1.2/x0.9/x1.1, print +0.1 ev."""
    th = default_theta(tab) + np.array([0.2, -0.1, 0.15, 0.05, -0.04, 0.03, 0.05, -0.06, 0.04, 0, 0, 0, 0.1])
    th[9:12] *= np.array([1.2, 0.9, 1.1])
    return th


def used_parameters(tab: dict) -> list:
    """Indices of the parameters the chain depends on for this record: the donor knees
    only with negative-donor DIR, the print gammas and print ev only on the print route."""
    used = list(range(6))
    if tab["dir_mode"] == 1:
        used += [9, 10, 11]
    if tab["print"]:
        used += [6, 7, 8, 12]
    return sorted(used)


def exposure(record, src, threads: int = 8) -> np.ndarray:
    """Camera exposure planes B, G, R (3, H, W) with the route correction: the oracle's
    FP32 film exposure, the input of the parameterised chain."""
    planes, _ = _orc.render(record, src, stage=6, threads=threads)
    return np.stack(planes)


def linear_rgb(record, src, threads: int = 8) -> np.ndarray:
    """The oracle's FP32 render to linear output RGB planes (3, H, W)."""
    planes, _ = _orc.render(record, src, stage=7, threads=threads)
    return np.stack(planes)


def _langmuir(torch, v, k, r):
    return v * (k + r) / (k + v)


def _curve(torch, x, y, q):
    """Piecewise-linear curve through (x, y) at q: the end values outside [x0, x_last],
    the interval whose right abscissa is the first one strictly above q inside
    (src/Cuda/JuicerCudaDeviceHelpers.cuh:34-89). x may carry gradients (the DIR axes)."""
    last = x.shape[0] - 1
    xd = x.detach()
    i1 = torch.searchsorted(xd, q.detach().contiguous(), right=True).clamp(1, last)
    i0 = i1 - 1
    x0, x1, y0, y1 = x[i0], x[i1], y[i0], y[i1]
    t = (q - x0) / (x1 - x0)
    v = y0 + t * (y1 - y0)
    v = torch.where(q <= xd[0], y[0].expand_as(v), v)
    return torch.where(q >= xd[last], y[last].expand_as(v), v)


def _coord(torch, nrm, res):
    top = float(res - 1)
    coord = (nrm * top).clamp(0.0, top)
    base = torch.floor(coord.detach()).clamp(max=res - 2).long()
    return base, coord - base.to(coord.dtype)


def _herm(y0, y1, m0, m1, t):
    t2 = t * t
    t3 = t2 * t
    return (2 * t3 - 3 * t2 + 1) * y0 + (t3 - 2 * t2 + t) * m0 + (-2 * t3 + 3 * t2) * y1 + (t3 - t2) * m1


def _lerp(a, b, t):
    return a + t * (b - a)


def _scan_lut(torch, lut, nd):
    """The scanner's PCHIP LUT at normalised densities nd (3, N): log2 X, Y, Z (3, N)
    (src/Cuda/JuicerCudaDeviceHelpers.cuh:357-506), clamped to the cell's range."""
    r = lut["res"]
    c, tc = _coord(torch, nd[0], r)
    m, tm = _coord(torch, nd[1], r)
    y, ty = _coord(torch, nd[2], r)
    s = r - 1
    outs = []
    for o in range(3):
        def at(tab, dc, dm, dy):
            return tab[(((c + dc) * r + (m + dm)) * r + (y + dy)) * 3 + o]

        v, sc, sm, sy = lut["v"], lut["sc"], lut["sm"], lut["sy"]
        v000 = _herm(at(v, 0, 0, 0), at(v, 1, 0, 0), at(sc, 0, 0, 0), at(sc, 1, 0, 0), tc)
        v010 = _herm(at(v, 0, 1, 0), at(v, 1, 1, 0), at(sc, 0, 1, 0), at(sc, 1, 1, 0), tc)
        v001 = _herm(at(v, 0, 0, 1), at(v, 1, 0, 1), at(sc, 0, 0, 1), at(sc, 1, 0, 1), tc)
        v011 = _herm(at(v, 0, 1, 1), at(v, 1, 1, 1), at(sc, 0, 1, 1), at(sc, 1, 1, 1), tc)
        sm00 = _lerp(at(sm, 0, 0, 0), at(sm, 1, 0, 0), tc)
        sm10 = _lerp(at(sm, 0, 1, 0), at(sm, 1, 1, 0), tc)
        sm01 = _lerp(at(sm, 0, 0, 1), at(sm, 1, 0, 1), tc)
        sm11 = _lerp(at(sm, 0, 1, 1), at(sm, 1, 1, 1), tc)
        vy0 = _herm(v000, v010, sm00, sm10, tm)
        vy1 = _herm(v001, v011, sm01, sm11, tm)
        sy0 = _lerp(_lerp(at(sy, 0, 0, 0), at(sy, 1, 0, 0), tc), _lerp(at(sy, 0, 1, 0), at(sy, 1, 1, 0), tc), tm)
        sy1 = _lerp(_lerp(at(sy, 0, 0, 1), at(sy, 1, 0, 1), tc), _lerp(at(sy, 0, 1, 1), at(sy, 1, 1, 1), tc), tm)
        val = _herm(vy0, vy1, sy0, sy1, ty)
        ci = ((c * s + m) * s + y) * 3 + o
        outs.append(torch.minimum(lut["hi"][ci], torch.maximum(lut["lo"][ci], val)))
    return torch.stack(outs)


class Chain:
    """The parameterised chain on one record, FP64, on `device` (CPU by default)."""

    def __init__(self, torch, record, oracle_module=None, device="cpu"):
        self.torch = torch
        tab = tables(record)
        self.tab = tab
        orc = oracle_module or _orc
        lut = orc.scanner_lut_for(record)
        d = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=device)  # noqa: E731
        names = ("v", "sc", "sm", "sy", "lo", "hi")
        self.lut = {k: d(np.asarray(a).ravel()) for k, a in zip(names, lut)}
        self.lut["res"] = tab["res"]
        self.t = {k: (d(v) if isinstance(v, np.ndarray) else v) for k, v in tab.items()}
        self.device = device

    def axes(self, k):
        """DIR compensated axes (3, n) for donor knees k (B, G, R): log exposure minus
        the coupler-matrix sum of the Langmuir donors of the curve densities."""
        torch, t = self.torch, self.t
        m = t["dir_m"].reshape(3, 3)  # [donor][receiver]
        if t["dir_mode"] == 2:
            # positive stocks: donors dmax - density, the receivers' Langmuir on the sums
            # (film/dir.rs:271-299); the knees do not enter
            c = m.T @ (t["dir_dmax"][:, None] - t["density_bgr"])
            cref, kr = t["dir_rcref"][:, None], t["dir_rkr"][:, None]
            fin = torch.where(cref == 0.0, torch.zeros_like(c), c * (kr + cref) / (kr + c))
            return t["log_exposure"][None, :] - fin
        donors = _langmuir(torch, t["density_bgr"], k[:, None], t["dir_dref"][:, None])  # (3 donor, n)
        return t["log_exposure"][None, :] - (m.T @ donors)

    def __call__(self, e0, theta, spatial=None):
        """e0: camera exposure (3, N) B, G, R (float64 tensor); theta (13,) float64.
        Returns the linear output RGB (3, N) (NaN where the LUT rejects a pixel).
        spatial: the spatial DIR filter, a differentiable map of the donor corrections
        of the B, G, R receivers (3, N) to the filtered corrections the development
        subtracts (src/Cuda/JuicerCudaDeviceHelpers.cuh:1267-1328); None for runtime
        DIR, where each pixel subtracts its own corrections."""
        torch, t = self.torch, self.t
        ev, gam, pgam, k, pev = theta[0:3], theta[3:6], theta[6:9], theta[9:12], theta[12]
        e = e0 * torch.exp2(ev)[:, None]
        logs = torch.log10(e.clamp(min=0.0) + 1e-10)
        x = t["log_exposure"]
        layer = torch.stack([_curve(torch, x, t["density_bgr"][c], logs[c] * gam[c]) for c in range(3)])
        if t["dir_mode"] == 1:
            donor = _langmuir(torch, layer, k[:, None], t["dir_dref"][:, None])
            m = t["dir_m"].reshape(3, 3)
            corr = m.T @ donor
            if spatial is not None:
                corr = spatial(corr)
            logc = logs - corr
            ax = self.axes(k)
            dens_bgr = [_curve(torch, ax[j], t["density_bgr"][j], logc[j] * gam[j]) for j in range(3)]
        elif t["dir_mode"] == 2:
            # positive stocks: donors are the density still to form; the receivers'
            # Langmuir finalises the (filtered) coupler sums
            # (src/Cuda/JuicerCudaDeviceHelpers.cuh:1173-1200)
            donor = t["dir_dmax"][:, None] - layer
            m = t["dir_m"].reshape(3, 3)
            corr = m.T @ donor
            if spatial is not None:
                corr = spatial(corr)
            cref, kr = t["dir_rcref"][:, None], t["dir_rkr"][:, None]
            fin = corr * (kr + cref) / (kr + corr)
            corr = torch.where(cref == 0.0, torch.zeros_like(fin), fin)
            logc = logs - corr
            ax = t["axes_bgr"]
            dens_bgr = [_curve(torch, ax[j], t["density_bgr"][j], logc[j] * gam[j]) for j in range(3)]
        elif t["dir_mode"] == 0:
            dens_bgr = [layer[c] for c in range(3)]
        else:
            raise ValueError("unknown DIR mode")
        dens = torch.stack([dens_bgr[2], dens_bgr[1], dens_bgr[0]])  # C, M, Y
        if t["print"]:
            sens = t["sens_cmy"]
            valid = ~torch.isnan(sens)
            sens0 = torch.where(valid, sens, torch.zeros_like(sens))
            dl = t["eps_cmy"] @ dens + t["base"][:, None]  # (81, N)
            tr = torch.pow(10.0, -dl) * t["illuminant"][:, None]
            raw = sens0.T @ tr  # (3, N)
            v = raw * t["midgray"]
            if t["preflash"] > 0.0:
                v = v + t["preflash_raw"][:, None] * t["preflash"]
            v = v * t["print_exposure"] * torch.exp2(pev) * t["print_route"]
            lp = torch.log10(v + 1e-10)
            px = t["print_log_exposure"]
            dens = torch.stack([_curve(torch, px, t["print_density_cmy"][c], lp[c] * pgam[c]) for c in range(3)])
        sign = 1.0 if t["medium_negative"] else -1.0
        nd = (dens + sign * t["min_cmy"][:, None]) * t["inv_cmy"][:, None]
        l2 = _scan_lut(torch, self.lut, nd)
        xyz = torch.exp2(l2)
        if t["corr_active"]:
            tt = t["corr_slope"] * xyz[1] + t["corr_offset"]
            cy = tt.clamp(0.0, 1.0)
            xyz = xyz * (cy / (xyz[1] + 1e-10))[None, :]
        ad = t["cat02"].reshape(3, 3) @ xyz
        return t["xyz_to_rgb"].reshape(3, 3) @ ad
