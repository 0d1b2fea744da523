"""Host-side recipe preparation: film/paper profiles -> the tables of FjPreparedHostData.

In Film-Juicer this precompute is Rust (rust/film-juicer-core/src/**, not buildable
here). This module restates the parts the render path consumes, in NumPy FP64, and
packs them into the same C-ABI record the Rust host fills:

* sensitivity: 10**log_sensitivity, non-finite -> 0 (exposure.rs:125-190, no band-pass);
* TC LUT: 192x192x81 Hanatos irradiance spectra contracted with the sensitivity,
  R,G,B,pad per node (reconstruction.rs:594-677; no spectral blur, no surface
  correction, no input-compression remap);
* density curves: the profile's curves (the Gaussian density model where the profile
  has one) minus their per-channel minimum, f32 (film.rs:72-93);
* DIR couplers: the reference's capture recipe at the stock gammas (dir_prep:
  film/dir.rs:135-365): coupler matrix, Langmuir knees and compensated log-exposure
  axes, pinned on the reference's DIR characterization;
* print: negative dye spectra, paper sensitivity (10^log in f32, non-finite -> 0),
  the TH-KG3 enlarger lamp through the dichroics at the calibrated neutral
  filtration, the preflash illuminant and raw integral, and the mid-grey balance
  normaliser of the film's reference densities (print_prep: print.rs:120-658,
  illuminant.rs:97-408, word for word; the reference densities come from this
  module's film tables);
* scanner: medium dye spectra with illuminant-weighted CIE 1931 CMFs
  (scanner.rs), density bounds of the medium;
* output: CAT02 from the viewing illuminant to D65, XYZ->linear sRGB, sRGB CCTF,
  OkLch gamut boundary 64x720 of the sRGB cube (gamut.rs:760, by bisection).

Where the restatement simplifies the Rust model it is stated above; the render
kernels consume whatever tables the host prepares, so parity of the render path
does not depend on these simplifications.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import abi, dir_prep, print_prep

WAVELENGTHS = np.arange(380.0, 781.0, 5.0)
N_LAMBDA = 81
LOG2_10 = math.log2(10.0)

# Linear Rec.709 / sRGB (D65) <-> CIE XYZ.
SRGB_TO_XYZ = np.array([[0.4123907992659595, 0.3575843393838780, 0.1804807884018343],
                        [0.2126390058715104, 0.7151686787677559, 0.0721923153607337],
                        [0.0193308187155918, 0.1191947797946259, 0.9505321522496606]])
XYZ_TO_SRGB = np.linalg.inv(SRGB_TO_XYZ)
CAT02 = np.array([[0.7328, 0.4296, -0.1624], [-0.7036, 1.6975, 0.0061], [0.0030, 0.0136, 0.9834]])
D65_XYZ = np.array([0.95047, 1.0, 1.08883])
D60_XYZ = np.array([0.95265, 1.0, 1.00883])
# RGB -> XYZ of the host's input colour spaces (published primaries; FJ_INPUT_* order)
INPUT_RGB_TO_XYZ = {
    0: np.array([[0.70062239, 0.14877482, 0.10105872], [0.27411851, 0.87363190, -0.14775041],
                 [-0.09896291, -0.13789533, 1.32591599]]),            # DaVinci Wide Gamut
    1: np.array([[0.6369580, 0.1446169, 0.1688810], [0.2627002, 0.6779981, 0.0593017],
                 [0.0, 0.0280727, 1.0609851]]),                       # BT.2020
    2: np.array([[0.9525524, 0.0, 0.0000937], [0.3439664, 0.7281661, -0.0721325],
                 [0.0, 0.0, 1.0088252]]),                             # ACES2065-1 (AP0, D60)
}

OK_XYZ_TO_LMS = np.array([[0.8189330101, 0.3618667424, -0.1288597137],
                          [0.0329845436, 0.9293118715, 0.0361456387],
                          [0.0482003018, 0.2643662691, 0.6338517070]])
OK_LMS_ROOT_TO_LAB = np.array([[0.2104542553, 0.7936177850, -0.0040720468],
                               [1.9779984951, -2.4285922050, 0.4505937099],
                               [0.0259040371, 0.7827717662, -0.8086757660]])


def _nan_array(values) -> np.ndarray:
    return np.array([[np.nan if v is None else v for v in row] if isinstance(row, list) else
                     (np.nan if row is None else row) for row in values], dtype=np.float64)


def load_profile(path: str) -> dict:
    with open(path) as fh:
        d = json.load(fh)
    data = d["data"]
    out = {"info": d["info"]}
    for key in ("log_sensitivity", "channel_density", "base_density", "midscale_neutral_density",
                "log_exposure", "density_curves"):
        out[key] = _nan_array(data[key])
    if "density_curves_layers" in data:
        out["density_curves_layers"] = _nan_array(data["density_curves_layers"])
    if isinstance(data.get("density_curves_model"), dict):
        out["density_curves_model"] = data["density_curves_model"]
    return out


def density_model_samples(centers, amplitudes, sigmas, log_exposure, positive: bool = False):
    """The Gaussian-CDF density model of a profile (model_type "norm_cdfs") sampled on a
    log-exposure axis, as the reference's host evaluates it
    (rust/film-juicer-core/src/profile.rs:482-520): per channel c and layer l, in FP32,
    z = sign (E - center) / sigma, cdf = 0.5 erfc(-z / sqrt 2), value = amplitude cdf,
    totals summed over the layers in layer order. Coefficient matrices are
    [channel][layer] (f64, narrowed to f32); returns totals [n, 3] and layers
    [n, layer, channel], float32.

    The reference evaluates erfcf from the Rust libm crate (=0.2.15, a port of the
    musl / FreeBSD single-precision erfc); here erfc is evaluated in FP64 (scipy) and
    rounded to f32. On the reference's 19 235 frozen samples
    (tests/profile/fixtures/density-samples.bin) the results are within 4 ulp, 86 %
    bit-identical (tests/test_density_model.py)."""
    from scipy.special import erfc

    e = np.asarray(log_exposure, dtype=np.float64).astype(np.float32)
    sign = np.float32(-1.0 if positive else 1.0)
    inv_sqrt2 = np.float32(0.7071067811865475244)
    totals = np.zeros((e.size, 3), np.float32)
    layers = np.zeros((e.size, 3, 3), np.float32)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        for c in range(3):
            t = np.zeros(e.size, np.float32)
            for l in range(3):
                center = np.float32(centers[c][l])
                amplitude = np.float32(amplitudes[c][l])
                sigma = np.float32(sigmas[c][l])
                z = (sign * (e - center)) / sigma
                cdf = np.float32(0.5) * erfc(((-z) * inv_sqrt2).astype(np.float64)).astype(np.float32)
                v = amplitude * cdf
                layers[:, l, c] = v
                t = t + v
            totals[:, c] = t
    return totals, layers


def profile_density_curves(prof: dict):
    """(totals [n, 3], layers [n, layer, channel]) of a loaded profile: the Gaussian
    model on the profile's log-exposure axis when the profile carries one (what the
    reference's host hands over), else the authored curves with their minimum
    subtracted."""
    m = prof.get("density_curves_model")
    if m and m.get("model_type") == "norm_cdfs":
        positive = prof["info"].get("type") == "positive"
        return density_model_samples(m["centers"], m["amplitudes"], m["sigmas"], prof["log_exposure"], positive)
    curves = prof["density_curves"].astype(np.float64)
    curves = curves - np.nanmin(curves, axis=0, keepdims=True)
    layers = prof.get("density_curves_layers")
    return curves.astype(np.float32), (np.asarray(layers, np.float32) if layers is not None else None)


def load_spectrum_csv(path: str) -> np.ndarray:
    rows = np.loadtxt(path, delimiter=",")
    return np.interp(WAVELENGTHS, rows[:, 0], rows[:, 1])


def load_cmfs(path: str) -> np.ndarray:
    rows = np.loadtxt(path, delimiter=",")
    return np.stack([np.interp(WAVELENGTHS, rows[:, 0], rows[:, k]) for k in (1, 2, 3)], axis=1)


def cat02_matrix(src_white: np.ndarray, dst_white: np.ndarray) -> np.ndarray:
    s = CAT02 @ (src_white / src_white[1])
    d = CAT02 @ (dst_white / dst_white[1])
    return np.linalg.inv(CAT02) @ np.diag(d / s) @ CAT02


def spectrum_xyz(spd: np.ndarray, cmfs: np.ndarray) -> np.ndarray:
    xyz = cmfs.T @ spd
    return xyz / xyz[1]


def build_tc_lut(spectra: np.ndarray, sens_rgb: np.ndarray) -> np.ndarray:
    """192x192x81 irradiance spectra x 81x3 sensitivity -> 192x192x4 (R,G,B,0) float32."""
    flat = spectra.reshape(-1, N_LAMBDA).astype(np.float64)
    rgb = flat @ np.nan_to_num(sens_rgb, nan=0.0)
    out = np.zeros((spectra.shape[0] * spectra.shape[1], 4), dtype=np.float32)
    out[:, :3] = rgb.astype(np.float32)
    return out.reshape(spectra.shape[0], spectra.shape[1], 4)


def gamut_boundary_table(rows: int = 64, hues: int = 720, lmin: float = 0.02, lmax: float = 1.0) -> np.ndarray:
    """Maximum OkLab chroma inside the linear sRGB cube per (lightness, hue)."""
    lab_to_lms_root = np.linalg.inv(OK_LMS_ROOT_TO_LAB)
    lms_to_xyz = np.linalg.inv(OK_XYZ_TO_LMS)
    L = np.linspace(lmin, lmax, rows)[:, None]
    h = (np.arange(hues) / hues) * 2 * np.pi - np.pi
    cos_h, sin_h = np.cos(h)[None, :], np.sin(h)[None, :]

    def inside(c):
        lab = np.stack([np.broadcast_to(L, c.shape), c * cos_h, c * sin_h], axis=-1)
        lms = (lab @ lab_to_lms_root.T) ** 3
        rgb = lms @ lms_to_xyz.T @ XYZ_TO_SRGB.T
        return np.all((rgb >= -1e-7) & (rgb <= 1 + 1e-7), axis=-1)

    lo = np.zeros((rows, hues))
    hi = np.full((rows, hues), 0.5)
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        ok = inside(mid)
        lo = np.where(ok, mid, lo)
        hi = np.where(ok, hi, mid)
    return lo.astype(np.float32)


@dataclass
class PreparedRecipe:
    """Arrays and scalars of one prepared render recipe (all float32 where the ABI is)."""

    route: int
    arrays: dict = field(default_factory=dict)
    scalars: dict = field(default_factory=dict)

    def save(self, path: str) -> None:
        payload = {f"a_{k}": v for k, v in self.arrays.items()}
        payload["scalars"] = np.array(json.dumps(self.scalars))
        payload["route"] = np.array(self.route)
        np.savez_compressed(path, **payload)

    @classmethod
    def load(cls, path: str) -> "PreparedRecipe":
        z = np.load(path, allow_pickle=False)
        arrays = {k[2:]: np.ascontiguousarray(z[k]) for k in z.files if k.startswith("a_")}
        return cls(int(z["route"]), arrays, json.loads(str(z["scalars"])))


def prepare_recipe(resources: str, film: str, paper: str | None = None, *, dir_amount: float = 1.0,
                   lut_resolution: int = 17, gamut: bool = True, exposure_ev: float = 0.0) -> PreparedRecipe:
    """Builds a direct (paper=None) or print recipe from the profile directory `resources`."""
    prof = load_profile(os.path.join(resources, "profiles", f"{film}.json"))
    cmfs = load_cmfs(os.path.join(resources, "cie1931_2deg.csv"))
    d50 = load_spectrum_csv(os.path.join(resources, "illuminants", "D50.csv"))
    d65 = load_spectrum_csv(os.path.join(resources, "illuminants", "D65.csv"))
    ref_ill = load_spectrum_csv(os.path.join(resources, "illuminants",
                                             f"{prof['info'].get('reference_illuminant', 'D55')}.csv"))
    spectra = np.load(os.path.join(resources, "luts", "spectral_upsampling", "irradiance_xy_tc.npy"))

    sens = np.power(10.0, prof["log_sensitivity"])
    sens = np.where(np.isfinite(sens) & (sens > 0), sens, 0.0)
    tc = build_tc_lut(spectra, sens)

    # Route correction: an 18.4 % grey of the reference illuminant exposes to 1 on green.
    grey_xyz = 0.184 * spectrum_xyz(ref_ill, cmfs)
    tcx = grey_xyz[0] / grey_xyz.sum()
    tcy = grey_xyz[1] / grey_xyz.sum()
    qx, qy = (1 - tcx) ** 2, tcy / max(1 - tcx, 1e-10)
    ci, mi = int(round(qx * 191)), int(round(qy * 191))
    g_grey = grey_xyz.sum() * tc[ci, mi, 1]
    route_scale = float(1.0 / g_grey)

    log_e = prof["log_exposure"].astype(np.float64)
    model_totals, model_layers = profile_density_curves(prof)
    # the development's curves: the profile's curves minus their per-channel minimum,
    # in f32 (film.rs:72-93), the curves the reference hands to the device
    norm_curves, _, _, norm_hash = dir_prep.normalized_curves(model_totals)
    curves = norm_curves.astype(np.float64)
    n = log_e.size

    a: dict[str, np.ndarray] = {}
    s: dict = {}
    f32 = lambda x: np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    a["sensitivity_rgb"] = f32(sens)
    a["tc_lut"] = f32(tc)
    a["log_exposure"] = f32(log_e)
    a["density_rgb"] = f32(curves)
    if model_layers is not None:
        # sublayer curves [sample][layer][channel] (the grain's layer model)
        a["density_layers"] = f32(model_layers)
    s["route_correction_scale"] = route_scale
    s["manual_exposure_ev"] = exposure_ev
    # Mallett 2019 reconstruction tables (81 x 3 basis, the film's reference
    # illuminant) and the green mid-grey scale of rust/film-juicer-core/src/exposure.rs:236-249
    # (1 / sum_l 0.184 I(l) S_green(l), accumulated in FP64, stored as f32).
    basis_path = os.path.join(resources, "luts", "spectral_upsampling", "mallett2019_basis.npy")
    if os.path.exists(basis_path):
        a["mallett_basis"] = f32(np.load(basis_path))
        a["mallett_illuminant"] = f32(ref_ill)
        green = 0.0
        for i in range(a["mallett_illuminant"].size):
            green += 0.184 * float(a["mallett_illuminant"][i]) * float(a["sensitivity_rgb"][i, 1])
        s["mallett_green_scale"] = float(np.float32(1.0 / green))
    s["input_rgb_to_xyz"] = SRGB_TO_XYZ.ravel().tolist()
    s["xyz_to_linear_srgb"] = XYZ_TO_SRGB.ravel().tolist()

    # DIR couplers: the capture recipe at the stock gammas, amount `dir_amount`
    # (film/dir.rs:135-365); matrix [donor][receiver], RGB order.
    params = dir_prep.capture_defaults(active=dir_amount > 0)
    params.amount = dir_amount
    rec = dir_prep.DirRecipe(norm_curves, f32(log_e), prof["info"].get("type") == "positive", params,
                             dir_prep.processing_defaults(prof["info"]), norm_hash)
    s["dir_mode"] = int(rec.mode)
    s["dir_matrix_rgb"] = [float(v) for v in rec.matrix_rgb.ravel()]
    s["dir_dmax"] = [float(v) for v in rec.density_max_rgb]
    s["dir_dref"] = [float(v) for v in rec.density_ref_rgb]
    s["dir_donor_k"] = [float(v) for v in rec.donor_k_rgb]
    s["dir_receiver_c_ref"] = [float(v) for v in rec.receiver_c_ref_rgb]
    s["dir_receiver_kr"] = [float(v) for v in rec.receiver_kr_rgb]
    s["dir_diffusion_um"] = [float(v) for v in rec.diffusion]
    s["dir_hash"] = str(rec.hash)
    s["dir_axes_hash"] = str(rec.axes_hash)
    if rec.mode:
        a["dir_axes_rgb"] = f32(rec.axes_rgb)

    positive = prof["info"].get("type") == "positive"
    route = abi.FJ_ROUTE_POSITIVE_DIRECT if positive else abi.FJ_ROUTE_NEGATIVE_DIRECT
    medium_dyes = prof["channel_density"]
    medium_base = prof["base_density"]
    medium_curves = curves
    if paper is not None:
        route = abi.FJ_ROUTE_POSITIVE_PRINT if positive else abi.FJ_ROUTE_NEGATIVE_PRINT
        pp = load_profile(os.path.join(resources, "profiles", f"{paper}.json"))
        # The enlarger: the TH-KG3 lamp through the dichroics at the calibrated neutral
        # filtration of this paper / lamp / film (recipe.rs:1709-1741, print.rs:120-158),
        # the mid-grey balance of the film's reference densities under it (print.rs:435-523).
        with open(os.path.join(resources, "filters", "heat_absorbing", "schott", "KG3.csv")) as fh:
            lamp = print_prep.tungsten_kg3(print_prep.parse_csv_rows(fh.read()))
        lamp_key = print_prep.enlarger_illuminant()  # the host's default lamp control: TH-KG3
        neutral, calibrated = print_prep.neutral_cmy_cc(resources, pp["info"].get("stock", paper), lamp_key,
                                                        prof["info"].get("stock", film))
        main_cc, preflash_cc = print_prep.filters(neutral)
        main_ill = print_prep.filtered_illuminant(main_cc, lamp)
        preflash_ill = print_prep.filtered_illuminant(preflash_cc, lamp)
        psens = print_prep.linear_sensitivity(pp["log_sensitivity"])
        neg_dyes = f32(prof["channel_density"])  # NaN kept: those wavelengths transmit nothing
        neg_base = f32(prof["base_density"])
        # The film's reference densities: the metered 18.4 % grey at 0 EV and at the
        # manual exposure through the film's density curves (film/reference.rs:214-262).
        # The reference's reconstruction balances that grey, so the metered grey lands at
        # log exposure 0 in every channel (the reference's product records sit within
        # 2e-4 of it) and at log10(2^ev) when compensated.
        ax, cv = f32(log_e), f32(curves)
        ref_density = []
        for ev in (0.0, exposure_ev):
            q = print_prep.F32(math.log10(2.0 ** ev))
            ref_density.append(f32([print_prep.sample_density(q, ax, cv, c) for c in range(3)]))
        ref_hash = print_prep.hash_u64s([print_prep.f32_bits(v) for v in np.concatenate(ref_density)])
        balance = print_prep.Balance(ref_density[0], ref_density[1], ref_hash,
                                     print_prep.normalization_mode(True, True), neg_base, neg_dyes, psens, main_ill)
        preflash_raw = print_prep.preflash_raw(neg_base, preflash_ill, psens)
        ple = pp["log_exposure"].astype(np.float64)
        pcurves = profile_density_curves(pp)[0].astype(np.float64)
        a["print_film_density_cmy"] = neg_dyes
        a["print_film_base_density"] = neg_base
        a["print_sensitivity_cmy"] = f32(psens)
        a["print_log_exposure"] = f32(ple)
        a["print_density_cmy"] = f32(pcurves)
        a["print_main_illuminant"] = f32(main_ill)
        a["print_preflash_illuminant"] = f32(preflash_ill)
        s["print_exposure"] = 1.0
        s["print_normalizer"] = float(balance.normalizer)
        s["print_reference_density_cmy"] = [[float(v) for v in d] for d in ref_density]
        s["print_main_cc_cmy"] = [float(v) for v in main_cc]
        s["print_preflash_cc_cmy"] = [float(v) for v in preflash_cc]
        s["print_neutral_calibrated"] = bool(calibrated)
        s["print_preflash_raw_cmy"] = [float(v) for v in preflash_raw]
        s["print_balance_hash"] = str(balance.hash)
        s["print_main_illuminant_hash"] = str(balance.filtered_main_illuminant_hash)
        s["print_preflash_illuminant_hash"] = str(print_prep.hash_finite_f32s(preflash_ill) or 0)
        s["print_preflash_raw_hash"] = str(print_prep.hash_finite_f32s(preflash_raw) or 0)
        medium_dyes = pp["channel_density"]
        medium_base = pp["base_density"]
        medium_curves = pcurves

    # Scanner: medium dye spectra under the D50 viewing illuminant.
    view = d50
    w = cmfs * view[:, None]
    inv_yn = float(1.0 / np.sum(w[:, 1]))
    a["scan_dye_c"] = f32(np.nan_to_num(medium_dyes[:, 0], nan=0.0))
    a["scan_dye_m"] = f32(np.nan_to_num(medium_dyes[:, 1], nan=0.0))
    a["scan_dye_y"] = f32(np.nan_to_num(medium_dyes[:, 2], nan=0.0))
    a["scan_wx"] = f32(w[:, 0])
    a["scan_wy"] = f32(w[:, 1])
    a["scan_wz"] = f32(w[:, 2])
    a["scan_base"] = f32(np.nan_to_num(medium_base, nan=0.0))
    s["scan_inv_yn"] = inv_yn
    # Density planes are C, M, Y; curve column k (the R, G, B sensitive layer) forms dye k.
    dmin = np.zeros(3)
    dspan = np.nanmax(medium_curves, axis=0)
    s["scan_min_cmy"] = dmin.tolist()
    s["scan_inv_span_cmy"] = (1.0 / (dspan * 1.05)).tolist()
    s["scan_lut_resolution"] = int(lut_resolution)
    view_xyz = spectrum_xyz(view, cmfs)
    s["cat02"] = cat02_matrix(view_xyz, D65_XYZ).ravel().tolist()
    s["xyz_to_rgb"] = XYZ_TO_SRGB.ravel().tolist()
    s["illuminant_xyz"] = view_xyz.tolist()
    s["gamut"] = bool(gamut)
    a["gamut_cmax"] = gamut_boundary_table()
    s["gamut_native_to_xyz"] = SRGB_TO_XYZ.ravel().tolist()
    s["gamut_xyz_to_native"] = XYZ_TO_SRGB.ravel().tolist()
    return PreparedRecipe(route, a, s)


class HostRecord:
    """An FjPreparedHostData filled from a PreparedRecipe; keeps every array alive."""

    def __init__(self, recipe: PreparedRecipe, *, recipe_hash: int = 0, auto_exposure: bool = False,
                 gamut: bool | None = None, dir_active: bool | None = None, correction=None,
                 method: int = abi.FJ_RAW_HANATOS_2025, input_space: int = abi.FJ_INPUT_SRGB_REC709,
                 decode: bool = False, adapt: bool = False, encoding: dict | None = None):
        """method: FJ_RAW_* (Mallett needs the recipe's Mallett tables); input_space,
        decode, adapt: the input colour space (FJ_INPUT_*), its CCTF decoding and the
        XYZ adaptation (to D65 for the D60 ACES white); encoding: an output-encoding
        entry of tests/golden/output_encoding_cases.json (colour space index, CCTF kind,
        parameters and DWG-to-output matrix as f32 words), encoded from DWG (the
        input-is-output flag cleared)."""
        self.recipe = recipe
        self._keep = []
        a, s = recipe.arrays, recipe.scalars
        h = abi.FjPreparedHostData()
        self.h = h
        h.route = recipe.route
        h.capture_polarity = abi.FJ_POLARITY_NEGATIVE
        h.recipe_hash = recipe_hash

        def span(arr):
            arr = np.ascontiguousarray(arr, dtype=np.float32)
            self._keep.append(arr)
            return abi.FjFloatSpan(arr.ctypes.data_as(C.POINTER(C.c_float)), arr.size)

        ex = h.film_exposure
        ex.input_color_space = input_space
        ex.method = method
        ex.flags = (abi.FJ_FILM_AUTO_EXPOSURE if auto_exposure else 0) | (abi.FJ_FILM_DECODE_CCTF if decode else 0) \
            | (abi.FJ_FILM_ADAPT_INPUT if adapt else 0)
        ex.manual_exposure_ev = s.get("manual_exposure_ev", 0.0)
        ex.route_correction_scale = s["route_correction_scale"]
        ex.mallett_green_midgray_scale = 1.0
        if input_space in INPUT_RGB_TO_XYZ:
            abi.set_floats(ex.input_rgb_to_xyz, INPUT_RGB_TO_XYZ[input_space].ravel())
        else:
            abi.set_floats(ex.input_rgb_to_xyz, s["input_rgb_to_xyz"])
        abi.set_floats(ex.input_xyz_adapt, (cat02_matrix(D60_XYZ, D65_XYZ) if adapt else np.eye(3)).ravel())
        if method == abi.FJ_RAW_MALLETT_2019:
            if "mallett_basis" not in a:
                raise ValueError("the recipe has no Mallett tables")
            ex.mallett_basis = span(a["mallett_basis"])
            ex.mallett_illuminant = span(a["mallett_illuminant"])
            ex.mallett_green_midgray_scale = s["mallett_green_scale"]
        abi.set_floats(ex.xyz_to_linear_srgb, s["xyz_to_linear_srgb"])
        ex.sensitivity_rgb = span(a["sensitivity_rgb"])
        ex.tc_lut_rgba = span(a["tc_lut"])
        ex.sensitivity_hash = ex.tc_lut_hash = ex.hash = 1

        dv = h.film_development
        dv.log_exposure = span(a["log_exposure"])
        dv.density_rgb = span(a["density_rgb"])
        if "density_layers" in a:
            for layer in range(3):
                for ch in range(3):
                    dv.density_layers[layer][ch] = span(a["density_layers"][:, layer, ch])
        abi.set_floats(dv.gamma_rgb, [1.0, 1.0, 1.0])
        dv.density_curves_hash = dv.hash = 1

        dmode = s.get("dir_mode", 0)
        if dir_active is False:
            dmode = 0
        dr = h.dir_couplers
        dr.mode = dmode
        if dmode:
            abi.set_floats(dr.matrix_rgb, s["dir_matrix_rgb"])
            abi.set_floats(dr.density_max_rgb, s["dir_dmax"])
            abi.set_floats(dr.density_ref_rgb, s["dir_dref"])
            abi.set_floats(dr.donor_k_rgb, s["dir_donor_k"])
            abi.set_floats(dr.receiver_c_ref_rgb, s.get("dir_receiver_c_ref", [0.0] * 3))
            abi.set_floats(dr.receiver_kr_rgb, s.get("dir_receiver_kr", [0.0] * 3))
            for c in range(3):
                dr.compensated_axes_rgb[c] = span(a["dir_axes_rgb"][c])
            dr.compensated_axes_hash = int(s.get("dir_axes_hash", 1)) or 1
            dr.hash = int(s.get("dir_hash", 1)) or 1

        sb = h.scanner_bounds
        abi.set_floats(sb.min_cmy, s["scan_min_cmy"])
        abi.set_floats(sb.inv_span_cmy, s["scan_inv_span_cmy"])
        sb.hash = 1
        sp = h.scanner_spectra
        sp.dye_c = span(a["scan_dye_c"])
        sp.dye_m = span(a["scan_dye_m"])
        sp.dye_y = span(a["scan_dye_y"])
        sp.weighted_x = span(a["scan_wx"])
        sp.weighted_y = span(a["scan_wy"])
        sp.weighted_z = span(a["scan_wz"])
        sp.base_density = span(a["scan_base"])
        sp.inverse_y_normalization = s["scan_inv_yn"]
        h.scanner_lut.resolution = s["scan_lut_resolution"]
        h.scanner_lut.hash = h.scanner_lut.density_bounds_hash = 1
        cr = h.scanner_correction
        cr.exposure_scale = 1.0
        cr.xyz_slope = 1.0
        if correction is not None:
            cr.flags = abi.FJ_CORRECTION_ACTIVE
            cr.xyz_slope, cr.xyz_offset = correction

        oc = h.output_color
        abi.set_floats(oc.cat02, s["cat02"])
        abi.set_floats(oc.xyz_to_rgb, s["xyz_to_rgb"])
        abi.set_floats(oc.illuminant_xyz, s["illuminant_xyz"])
        oc.color_space = abi.FJ_OUTPUT_SRGB
        use_gamut = s.get("gamut", True) if gamut is None else gamut
        oc.flags = abi.FJ_COLOR_ENCODE_CCTF | abi.FJ_COLOR_INPUT_IS_OUTPUT_SPACE | (
            abi.FJ_COLOR_GAMUT_COMPRESSION if use_gamut else 0)
        abi.set_floats(oc.native_rgb_to_d65_xyz, s["gamut_native_to_xyz"])
        abi.set_floats(oc.d65_xyz_to_native_rgb, s["gamut_xyz_to_native"])
        abi.set_floats(oc.lightness_knee, [0.95, 1.0, 1.6])
        abi.set_floats(oc.chroma_knee, [0.95, 1.0, 1.6])
        oc.gamut_cmax = span(a["gamut_cmax"])
        oc.encoding.schema = abi.FJ_OUTPUT_ENCODING_SCHEMA
        oc.encoding.cctf_kind = abi.FJ_CCTF_SRGB
        oc.encoding.gamma = 1.0 / 2.4
        abi.set_floats(oc.encoding.dwg_to_output, np.eye(3).ravel())
        if encoding is not None:
            f = lambda w: float(np.array([w], np.uint32).view(np.float32)[0])  # noqa: E731
            oc.color_space = encoding["color_space"]
            oc.flags &= ~abi.FJ_COLOR_INPUT_IS_OUTPUT_SPACE
            en = oc.encoding
            en.cctf_kind = encoding["cctf_kind"]
            en.gamma, en.a, en.b, en.c, en.d, en.linear_cutoff = (f(w) for w in encoding["params"])
            abi.set_floats(en.dwg_to_output, [f(w) for w in encoding["dwg_to_output"]])

        if recipe.route in (abi.FJ_ROUTE_NEGATIVE_PRINT, abi.FJ_ROUTE_POSITIVE_PRINT):
            pr = h.print
            pr.film_density_cmy = span(a["print_film_density_cmy"])
            pr.film_base_density = span(a["print_film_base_density"])
            pr.sensitivity_cmy = span(a["print_sensitivity_cmy"])
            pr.log_exposure = span(a["print_log_exposure"])
            pr.density_cmy = span(a["print_density_cmy"])
            pr.main_illuminant = span(a["print_main_illuminant"])
            pr.exposure = s["print_exposure"]
            pr.normalizer = s["print_normalizer"]
            pr.hash = pr.film_density_hash = pr.profile_tables_hash = 1
            pr.balance_hash = pr.main_illuminant_hash = 1
            if "print_preflash_illuminant" in a:
                pr.preflash_illuminant = span(a["print_preflash_illuminant"])
                abi.set_floats(pr.main_cc_cmy, s["print_main_cc_cmy"])
                abi.set_floats(pr.preflash_cc_cmy, s["print_preflash_cc_cmy"])
                abi.set_floats(pr.preflash_raw_cmy, s["print_preflash_raw_cmy"])
                pr.balance_hash = int(s["print_balance_hash"])
                pr.main_illuminant_hash = int(s["print_main_illuminant_hash"])
                pr.preflash_illuminant_hash = int(s["print_preflash_illuminant_hash"])
                pr.preflash_raw_hash = int(s["print_preflash_raw_hash"])
                pr.preflash_exposure = float(s.get("print_preflash_exposure", 0.0))
                if pr.preflash_exposure > 0.0:
                    pr.flags |= abi.FJ_PRINT_PREFLASH

        ae = h.auto_exposure
        ae.method = abi.FJ_METER_CENTER_WEIGHTED
        ae.hash = 1

    def pointer(self):
        return C.pointer(self.h)


def synthetic_frame(width: int, height: int, seed: int, frame_index: int = 0) -> np.ndarray:
    """Seeded smooth test scene, float32 linear Rec.709 RGB, shape (height, width, 3).

    Three fields u1, u2, u3 in [0, 1], each 0.5 * a linear ramp at a random angle plus
    0.5 * a sum of 16 Gaussian blobs (sigma 2-12 % of the width), normalised;
    log2 Y = -8 + 12 u1, hue = 2 pi u2, chroma = 0.3 u3; RGB = Y (1 + chroma
    (cos h a + sin h b)) with a, b unit opponent axes orthogonal to the Rec.709
    luminance weights; negatives clamped to zero.
    """
    rng = np.random.Generator(np.random.PCG64(seed + frame_index))
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float32)
    xn, yn = xx / max(width, 1), yy / max(width, 1)

    def field_():
        ang = rng.uniform(0, 2 * np.pi)
        ramp = np.cos(ang) * xn + np.sin(ang) * yn
        ramp = (ramp - ramp.min()) / max(float(np.ptp(ramp)), 1e-6)
        blobs = np.zeros_like(xn)
        for _ in range(16):
            cx, cy = rng.uniform(0, 1), rng.uniform(0, height / max(width, 1))
            sg = rng.uniform(0.02, 0.12)
            blobs += rng.uniform(0.2, 1.0) * np.exp(-((xn - cx) ** 2 + (yn - cy) ** 2) / (2 * sg * sg))
        blobs = (blobs - blobs.min()) / max(float(np.ptp(blobs)), 1e-6)
        f = 0.5 * ramp + 0.5 * blobs
        return (f - f.min()) / max(float(np.ptp(f)), 1e-6)

    u1, u2, u3 = field_(), field_(), field_()
    lum = np.exp2(-8.0 + 12.0 * u1)
    hue = 2 * np.pi * u2
    chroma = 0.3 * u3
    wts = np.array([0.2126, 0.7152, 0.0722])
    a_ax = np.array([1.0, -1.0, 0.0])
    a_ax -= wts * (a_ax @ wts) / (wts @ wts)
    a_ax /= np.linalg.norm(a_ax)
    b_ax = np.cross(wts, a_ax)
    b_ax -= wts * (b_ax @ wts) / (wts @ wts)
    b_ax /= np.linalg.norm(b_ax)
    mod = 1.0 + chroma[..., None] * (np.cos(hue)[..., None] * a_ax + np.sin(hue)[..., None] * b_ax)
    rgb = lum[..., None] * mod
    return np.ascontiguousarray(np.maximum(rgb, 0.0).astype(np.float32))


# ---------------------------------------------------------------------------
# Scatter / halation descriptor (rust/film-juicer-core/src/optics/halation_frame.rs)
# ---------------------------------------------------------------------------
HALATION_TAIL_RATIOS = (0.5360, 1.5236, 2.7684)
HALATION_BOUNCE_MULTIPLIERS = (1.0, 1.4142135623730950488, 1.7320508075688772935, 2.0, 2.23606797749979)


def _yvv_coefficients(sigma: float):
    """Young-van Vliet third-order coefficients [B, b1/b0, b2/b0, b3/b0] (halation_frame.rs:221-229)."""
    q = 0.98711 * sigma - 0.96330
    q2, q3 = q * q, q * q * q
    b0 = 1.57825 + 2.44413 * q + 1.4281 * q2 + 0.422205 * q3
    b1 = 2.44413 * q + 2.85619 * q2 + 1.26661 * q3
    b2 = -(1.4281 * q2 + 1.26661 * q3)
    b3 = 0.422205 * q3
    return [1.0 - (b1 + b2 + b3) / b0, b1 / b0, b2 / b0, b3 / b0]


def _factored(coeffs):
    """Real pole + second-order section factors [h, g, t, 0] (halation_frame.rs:88-146)."""
    b, a1, a2, a3 = coeffs
    c1 = 3.0 - 2.0 * a1 - a2
    c2 = 3.0 - a1
    poly = lambda h: ((-h + c2) * h - c1) * h + b
    lo, hi = 0.0, 1.0
    for _ in range(64):
        mid = (lo + hi) * 0.5
        if poly(mid) > 0.0:
            lo = mid
        else:
            hi = mid
    h = (lo + hi) * 0.5
    t = a3 / (1.0 - h)
    g = b / h
    return [np.float32(h), np.float32(g), np.float32(t), np.float32(0.0)]


def halation_gaussian(out: "abi.FjHalationGaussian", sigma_px: float, legacy: bool = True) -> None:
    """Fills one FjHalationGaussian the way halation_frame.rs:157-236 builds it."""
    C.memset(C.addressof(out), 0, C.sizeof(out))
    if not (sigma_px > 0.0):
        out.kind = abi.FJ_HALATION_IDENTITY
        return
    if sigma_px < 3.0:
        radius = int(3.0 * sigma_px + 0.5)
        if radius == 0:
            out.kind = abi.FJ_HALATION_IDENTITY
            return
        x = np.arange(-radius, radius + 1, dtype=np.float64)
        w = np.exp(-(x * x) / (2.0 * sigma_px * sigma_px))
        w = (w / w.sum()).astype(np.float32)
        out.kind = abi.FJ_HALATION_FIR_REFLECT
        out.radius = radius
        for i, v in enumerate(w):
            out.fir_weights[i] = float(v)
        return
    co = _yvv_coefficients(sigma_px)
    if legacy:
        out.kind = abi.FJ_HALATION_YVV_REPLICATE
        vals = [np.float32(v) for v in co]
    else:
        out.kind = abi.FJ_HALATION_YVV_REPLICATE_FACTORED
        vals = _factored(co)
    for i, v in enumerate(vals):
        out.yvv[i] = float(v)


def scatter_halation_record(pixel_size_um: float, *, scatter_amount: float = 0.35,
                            core_um=(14.0, 11.0, 8.0), tail_um=(60.0, 45.0, 30.0), tail_weight=(0.25, 0.2, 0.15),
                            halation_first_sigma_um=(90.0, 70.0, 50.0), strength=(0.08, 0.03, 0.0),
                            bounce_weights=(0.6, 0.25, 0.15), renormalize: bool = True,
                            legacy: bool = True) -> "abi.FjScatterHalation":
    """An FjScatterHalation for the given pixel size with plausible still-film settings
    (sigmas in micrometres; channels R, G, B)."""
    d = abi.FjScatterHalation()
    d.recipe_hash = 1
    d.scatter_amount = scatter_amount
    d.bounce_count = len(bounce_weights)
    for i, w in enumerate(bounce_weights):
        d.bounce_weights[i] = w
    d.renormalize = 1 if renormalize else 0
    for c in range(3):
        ch = d.channels[c]
        ch.tail_weight = tail_weight[c]
        ch.total_strength = strength[c]
        if ch.tail_weight != 1.0:
            halation_gaussian(ch.core, max(core_um[c] / pixel_size_um, 1e-6), legacy)
        if ch.tail_weight != 0.0:
            for i in range(3):
                halation_gaussian(ch.tail[i], max(tail_um[c] * HALATION_TAIL_RATIOS[i] / pixel_size_um, 1e-6), legacy)
        if ch.total_strength != 0.0:
            for b in range(d.bounce_count):
                halation_gaussian(ch.bounce[b], halation_first_sigma_um[c] * HALATION_BOUNCE_MULTIPLIERS[b]
                                  / pixel_size_um, legacy)
    return d
