"""Film and gate defects (the path's third next row): film dust and scratches on the
capture density, the gate mask, weave and the gate mask at the output encoding.

Records: the composed FjFilmEffects of the reference's effects-frame characterization
(tests/golden/effects_cases.json: activation, ROI offsets, negative and 2^31-scale
cell coordinates, weave, split grids), with the slot probabilities raised so that a
64 x 48 frame shows defects.

Against the reference's own CUDA launchers (juicer_cuda_apply_film_defects,
juicer_cuda_build_gate_defect_transmittance_focused, the focused scan and scanner
output launchers, compiled for sm_100a) on the same density planes: the dust plane,
the scratched densities and the gate mask bit for bit; the encoded frame within 1e-6
(direct route; the print route adds the print development's float rounding, 2e-5).
Against the oracle's restatement (libm's cosf/sinf/hypotf and no fused multiply-add,
so particle edges can move by a rounding): tolerance bounds on a pixel fraction."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [0, 1, 2, 18, 20, 25, 119, 168]
DUSTY = {0, 1, 18, 20, 25, 119}  # cases whose frame shows film dust at the raised slot probability


@pytest.fixture(scope="module")
def ref_lib(oracle):
    lib = oracle.load_reference()
    if lib is None or not hasattr(lib, "ref_effects_render"):
        pytest.skip("reference CUDA harness not built with the defects entry")
    return lib


def frame_size(e):
    return e.render_extent.width, e.render_extent.height


def density_planes(torch, dr, src):
    planes = [torch.empty(src.shape[:2], device="cuda") for _ in range(3)]
    dr.capture_density(torch.from_numpy(src).cuda(), planes)
    torch.cuda.synchronize()
    return planes


def mine_render(torch, runtime, descriptors, dr, e, dens, s):
    from film_juicer_b200 import abi

    dens = [d.clone() for d in dens]
    dust = runtime.film_defects(e, dens) if e.flags & abi.FJ_EFFECTS_FILM else None
    gate = (e.flags & abi.FJ_EFFECTS_GATE_OUTPUT) and (e.flags & abi.FJ_EFFECTS_GATE_TRANSMITTANCE)
    mask = runtime.gate_mask(e) if gate else None
    out = torch.full_like(s, -1.0)
    runtime.render_from_density_effects(dr, descriptors.scanner_post_record(hash=0), 0, (0, 0), e, dust, mask, dens,
                                        out, src=s)
    torch.cuda.synchronize()
    return dens, dust, mask, out


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("route", ["print", "direct"])
def test_defects_match_reference_cuda(torch_cuda, ref_lib, oracle, recipes, prepare, effects_case, route, case):
    torch = torch_cuda
    from film_juicer_b200 import abi, descriptors, runtime

    e = effects_case(case)
    w, h = frame_size(e)
    rec = prepare.HostRecord(recipes[route])
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=31 + case))
    s = torch.from_numpy(src).cuda()
    dr = runtime.DeviceRecipe(rec)
    dens = density_planes(torch, dr, src)
    m_dens, m_dust, m_mask, m_out = mine_render(torch, runtime, descriptors, dr, e, dens, s)

    r_dens = [d.clone() for d in dens]
    r_dust = torch.full((h, w), -1.0, device="cuda")
    r_mask = torch.full((max(e.gate_height, 1), max(e.gate_width, 1)), -1.0, device="cuda")
    r_out = torch.full_like(s, -1.0)
    lut = oracle.scanner_lut_for(rec)
    ptrs = (C.c_void_p * 6)(*[o.ctypes.data for o in lut])
    rc = ref_lib.ref_effects_render(rec.pointer(), ptrs, C.byref(e), *[C.c_void_p(p.data_ptr()) for p in r_dens],
                                    C.c_void_p(s.data_ptr()), w * 12, C.c_void_p(r_out.data_ptr()), w * 12, w, h, 3,
                                    C.c_void_p(r_dust.data_ptr()), C.c_void_p(r_mask.data_ptr()))
    assert rc == 0
    torch.cuda.synchronize()
    if e.flags & abi.FJ_EFFECTS_FILM:
        # the scratched capture density (scanned by the direct route, printed by the
        # print route: compare before the print -- the reference prints in place)
        if route == "direct":
            for a, b in zip(m_dens, r_dens):
                assert torch.equal(a, b)
        if m_dust is not None:
            assert torch.equal(m_dust, r_dust)
            if case in DUSTY:
                assert float(m_dust.min()) < 0.999
    if m_mask is not None:
        assert torch.equal(m_mask, r_mask)
        if case in DUSTY:
            assert float(m_mask.min()) < 0.999
    a, b = m_out.cpu().numpy(), r_out.cpu().numpy()
    assert np.all(np.isfinite(a))
    err = np.abs(a - b)
    bound = 1e-6 if route == "direct" else 2e-5
    assert float(err.max()) <= bound, (case, float(err.max()), float((err > 0).mean()))
    dr.close()


@pytest.mark.parametrize("case", [0, 18, 119])
def test_defects_match_oracle(torch_cuda, oracle, recipes, prepare, effects_case, case):
    torch = torch_cuda
    from film_juicer_b200 import abi, descriptors, runtime

    e = effects_case(case)
    w, h = frame_size(e)
    rec = prepare.HostRecord(recipes["print"])
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=7 + case))
    s = torch.from_numpy(src).cuda()
    dr = runtime.DeviceRecipe(rec)
    dens = density_planes(torch, dr, src)
    m_dens, m_dust, m_mask, m_out = mine_render(torch, runtime, descriptors, dr, e, dens, s)
    o_dens, o_dust = oracle.film_defects(e, [d.cpu().numpy() for d in dens])
    if m_dust is not None:
        err = np.abs(m_dust.cpu().numpy() - o_dust)
        assert float((err > 1e-4).mean()) <= 0.01 and float(err.max()) <= 0.05, (case, float(err.max()))
    for a, b in zip(m_dens, o_dens):
        err = np.abs(a.cpu().numpy() - b)
        assert float((err > 1e-4).mean()) <= 0.01 and float(err.max()) <= 0.05
    o_mask = None
    if (e.flags & abi.FJ_EFFECTS_GATE_OUTPUT) and (e.flags & abi.FJ_EFFECTS_GATE_TRANSMITTANCE):
        o_mask = oracle.gate_mask(e)
        err = np.abs(m_mask.cpu().numpy() - o_mask)
        assert float((err > 1e-4).mean()) <= 0.02 and float(err.max()) <= 0.05, (case, float(err.max()))
    # the output from the oracle's planes: only the scan and encoding differ
    want, _ = oracle.render_effects(rec, descriptors.scanner_post_record(hash=0), 0, 0, 0, e,
                                    m_dust.cpu().numpy() if m_dust is not None else None,
                                    m_mask.cpu().numpy() if m_mask is not None else None,
                                    [d.cpu().numpy() for d in m_dens], src=src)
    got = m_out.cpu().numpy()
    err = np.abs(got - want)
    bad = err > 2e-4 + 3e-4 * np.abs(want)
    assert float(bad.mean()) <= 0.01, (case, float(bad.mean()), float(err.max()))
    dr.close()


@pytest.mark.parametrize("route", ["print", "direct"])
def test_frame_schedule_with_effects_matches_oracle_chain(torch_cuda, recipes, prepare, effects_case, route):
    from film_juicer_b200 import frame_records, runtime
    from oracle import frame as oframe

    torch = torch_cuda
    e = effects_case(119)  # film dust and scratches, gate mask and weave
    w, h = frame_size(e)
    rec = frame_records.FrameRecord(recipes[route], w, h, effects=e)
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261207))
    s = torch.from_numpy(src).cuda()
    d = torch.full_like(s, -1.0)
    with runtime.Owner() as owner:
        owner.render(rec, s, d, frame_token=3)
    got = d.cpu().numpy()
    want, _ = oframe.render_frame(rec, recipes[route], src, frame_token=3)
    err = np.abs(got - want)
    bad = err > 2e-4 + 3e-4 * np.abs(want)
    assert float(bad.mean()) <= 0.02, (route, float(bad.mean()), float(err.max()))
    assert float(err.mean()) <= 2e-4, (route, float(err.mean()))


def test_effects_change_the_frame_and_inactive_records_do_not(torch_cuda, recipes, prepare, effects_case):
    from film_juicer_b200 import abi, frame_records, runtime

    torch = torch_cuda
    e = effects_case(0)
    w, h = frame_size(e)
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=5))
    s = torch.from_numpy(src).cuda()
    outs = []
    for fx in (None, abi.FjFilmEffects(), e):
        rec = frame_records.FrameRecord(recipes["print"], w, h, effects=fx)
        d = torch.full_like(s, -1.0)
        with runtime.Owner() as owner:
            owner.render(rec, s, d, frame_token=1)
        outs.append(d)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])
    assert float((outs[2] - outs[0]).abs().max()) > 1e-3


@pytest.mark.parametrize("case", [0, 18, 25, 119])
def test_particle_table_changes_no_result(torch_cuda, effects_case, case):
    # with the per-frame particle table or with each tile building its own candidates,
    # the dust plane, the scratched densities and the gate mask are the same bits
    from film_juicer_b200 import abi, runtime

    torch = torch_cuda
    e = effects_case(case)
    w, h = frame_size(e)
    g = torch.Generator(device="cuda").manual_seed(case)
    base = [torch.rand((h, w), device="cuda", generator=g) * 2.0 for _ in range(3)]
    a = [t.clone() for t in base]
    b = [t.clone() for t in base]
    da = runtime.film_defects(e, a, table=True)
    db = runtime.film_defects(e, b, table=False)
    torch.cuda.synchronize()
    assert all(torch.equal(x, y) for x, y in zip(a, b))
    assert (da is None and db is None) or torch.equal(da, db)
    if e.flags & abi.FJ_EFFECTS_GATE_TRANSMITTANCE:
        assert torch.equal(runtime.gate_mask(e, table=True), runtime.gate_mask(e, table=False))
