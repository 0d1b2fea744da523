"""Branches of the per-pixel chain that the default recipe does not take, against the
reference's own CUDA kernels (oracle/_ref) and the oracle, through fjb_render_pixels:

* Mallett 2019 reconstruction (81-wavelength basis x illuminant x sensitivity,
  src/Cuda/JuicerCudaDeviceHelpers.cuh:619), direct and print routes;
* input decoding and colour spaces (:198, :509, :537): sRGB and BT.2020 CCTF decoding,
  DaVinci Wide Gamut and ACES2065-1 primaries, the input XYZ adaptation;
* the nine output encodings of the reference's frozen table
  (tests/scanner/output_encoding_native.inc: linear, gamma, sRGB, BT.2020, ProPhoto
  and DaVinci Intermediate CCTFs with their DWG-to-output matrices;
  src/Cuda/Scan/JuicerCudaScanPipeline.cu:99-152), encoded from DWG.
Bound: the reference's processor-pixel bound 2e-4 + 3e-4 |ref| per encoded channel,
and equal error flags. The pure power CCTF (kind 1, v^gamma) has an unbounded slope at
black; for it the bound adds a linear-domain allowance of 4e-6 carried through the
CCTF's slope at the encoded value (OkLch gamut compression of a saturated colour
leaves a channel near zero as a difference of terms ~1e4 times larger, so FP32
implementations of it differ there by a few 1e-6 in linear light: the reference's
CUDA and the oracle differ by as much as this library does)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from film_juicer_b200 import abi

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLDEN, "output_encoding_cases.json")) as fh:
    ENCODINGS = json.load(fh)["entries"]
INPUTS = {"srgb_decode": (abi.FJ_INPUT_SRGB_REC709, True, False), "bt2020_decode": (abi.FJ_INPUT_BT2020, True, False),
          "dwg": (abi.FJ_INPUT_DWG, False, False), "dwg_decode_flag": (abi.FJ_INPUT_DWG, True, False),
          "aces_adapt": (abi.FJ_INPUT_ACES2065_1, False, True)}


@pytest.fixture(scope="module")
def ref_lib(oracle):
    lib = oracle.load_reference()
    if lib is None:
        pytest.skip("reference CUDA harness not built (needs the reference sources at build time)")
    return lib


def _cctf_allowance(rec, mine, ref):
    """Linear-domain allowance 4e-6 through the slope of a pure power CCTF (kind 1)."""
    if rec.h.output_color.encoding.cctf_kind != 1 or not (rec.h.output_color.flags & abi.FJ_COLOR_ENCODE_CCTF):
        return 0.0
    g = float(rec.h.output_color.encoding.gamma)
    y = np.maximum(np.maximum(np.abs(ref), np.abs(mine)), 1e-3).astype(np.float64)
    slope = g * np.power(y, (g - 1.0) / g)  # d(v^g)/dv at v = y^(1/g)
    return 4e-6 * slope


def _check(torch, ref_lib, oracle, rec, src):
    from film_juicer_b200 import runtime

    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    s = torch.from_numpy(src).cuda()
    ref_d = torch.zeros_like(s)
    rflags = C.c_uint32()
    h, w, comps = src.shape
    rc = ref_lib.ref_render(rec.pointer(), ptrs, C.c_void_p(s.data_ptr()), w * comps * 4,
                            C.c_void_p(ref_d.data_ptr()), w * comps * 4, w, h, comps, C.byref(rflags))
    assert rc == 0, f"reference launcher returned cudaError {rc}"
    ref = ref_d.cpu().numpy()
    dr = runtime.DeviceRecipe(rec)
    d = torch.empty_like(s)
    dr.clear_flags()
    dr.render(s, d)
    flags = dr.read_flags()
    dr.close()
    mine = d.cpu().numpy()
    orc, oflags = oracle.render(rec, src)
    assert flags == int(rflags.value) == oflags
    tol = 2e-4 + 3e-4 * np.abs(ref)
    tol = tol + _cctf_allowance(rec, mine, ref) + _cctf_allowance(rec, orc, ref)
    assert np.all(np.isfinite(mine))
    assert np.all(np.abs(mine - ref) <= tol), float(np.max(np.abs(mine - ref)))
    assert np.all(np.abs(orc - ref) <= tol), float(np.max(np.abs(orc - ref)))
    return mine


@pytest.mark.parametrize("route", ["direct", "print"])
@pytest.mark.parametrize("size", [(200, 120), (512, 512)])
def test_mallett_reconstruction(torch_cuda, ref_lib, oracle, recipes, prepare, route, size):
    rec = prepare.HostRecord(recipes[route], method=abi.FJ_RAW_MALLETT_2019)
    src = np.ascontiguousarray(prepare.synthetic_frame(*size, seed=20261203))
    out = _check(torch_cuda, ref_lib, oracle, rec, src)
    hanatos = _check(torch_cuda, ref_lib, oracle, prepare.HostRecord(recipes[route]), src)
    assert float(np.abs(out - hanatos).max()) > 1e-3  # a different reconstruction ran


@pytest.mark.parametrize("route", ["direct", "print"])
@pytest.mark.parametrize("name", list(INPUTS))
def test_input_decoding_and_spaces(torch_cuda, ref_lib, oracle, recipes, prepare, route, name):
    space, decode, adapt = INPUTS[name]
    rec = prepare.HostRecord(recipes[route], input_space=space, decode=decode, adapt=adapt)
    lin = prepare.synthetic_frame(160, 90, seed=41)
    # encoded-domain values for the decoding cases (a display-referred signal in 0..1.2)
    src = np.ascontiguousarray(np.power(np.clip(lin, 0.0, 1.5), 1.0 / 2.2).astype(np.float32) if decode else lin)
    src[0, 0] = [-0.25, 0.0, 2.0]  # negative and above-one channels through the decoders
    _check(torch_cuda, ref_lib, oracle, rec, src)


@pytest.mark.parametrize("route", ["direct", "print"])
@pytest.mark.parametrize("entry", ENCODINGS, ids=[f"space{e['color_space']}_cctf{e['cctf_kind']}" for e in ENCODINGS])
def test_output_encodings(torch_cuda, ref_lib, oracle, recipes, prepare, route, entry):
    rec = prepare.HostRecord(recipes[route], encoding=entry)
    src = np.ascontiguousarray(prepare.synthetic_frame(150, 80, seed=43))
    out = _check(torch_cuda, ref_lib, oracle, rec, src)
    assert float(out.min()) >= 0.0 and float(out.max()) <= 1.0
