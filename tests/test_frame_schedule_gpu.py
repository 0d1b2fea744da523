"""The drop-in fj_cuda_render with the whole staged schedule (camera exposure, camera
diffusion, scatter/halation, spatial DIR, capture density, grain, print, scan,
output) against the oracle's chain of the same stages.

Every stage agrees with its oracle to FP32 rounding (see the per-stage tests); grain
turns last-bit differences of its inputs into occasional one-particle differences,
which the later stages spread over a few pixels. The bound is therefore the
reference's pixel bound, 2e-4 + 3e-4 |oracle| per encoded channel, on at least 99 %
of the pixels, and a mean absolute difference below 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ATOL, RTOL = 2e-4, 3e-4


def run(torch, record, src):
    from film_juicer_b200 import runtime

    s = torch.from_numpy(src).cuda()
    d = torch.full_like(s, -1.0)
    with runtime.Owner() as owner:
        out = owner.render(record, s, d)
    return d.cpu().numpy(), out


CONFIGS = {
    "all_stages": dict(),
    "all_stages_auto_exposure": dict(auto_exposure=True),
    "grain_only": dict(diffusion=False, halation=False, spatial_dir=False),
    "optics_only": dict(spatial_dir=False, grain=False),
    "spatial_dir_only": dict(diffusion=False, halation=False, grain=False),
}


@pytest.mark.parametrize("name", list(CONFIGS))
@pytest.mark.parametrize("route", ["print", "direct"])
def test_frame_schedule_matches_oracle_chain(torch_cuda, recipes, prepare, route, name):
    from film_juicer_b200 import frame_records
    from oracle import frame as oframe

    w, h = 120, 72
    rec = frame_records.FrameRecord(recipes[route], w, h, **CONFIGS[name])
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=20261205))
    got, out = run(torch_cuda, rec, src)
    want, _ = oframe.render_frame(rec, recipes[route], src)
    assert np.all(np.isfinite(got))
    err = np.abs(got - want)
    bad = err > ATOL + RTOL * np.abs(want)
    assert float(bad.mean()) <= 0.01, (name, float(bad.mean()), float(err.max()))
    assert float(err.mean()) <= 1e-4, (name, float(err.mean()))


def test_auto_exposure_monolithic_matches_oracle(torch_cuda, recipes, prepare, oracle):
    from film_juicer_b200 import frame_records

    w, h = 96, 64
    rec = frame_records.FrameRecord(recipes["direct"], w, h, diffusion=False, halation=False, spatial_dir=False,
                                    grain=False, auto_exposure=True)
    src = np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=7)) * np.float32(5.0)
    got, _ = run(torch_cuda, rec, src)
    scale = oracle.auto_exposure(rec.host, rec.host.h.auto_exposure, src)
    want, _ = oracle.render(rec.host, src, auto_scale=scale)
    err = np.abs(got - want)
    assert np.all(err <= ATOL + RTOL * np.abs(want)), float(err.max())


def test_frame_schedule_is_deterministic_and_reuses_the_owner(torch_cuda, recipes, prepare):
    from film_juicer_b200 import frame_records, runtime

    torch = torch_cuda
    w, h = 64, 48
    rec = frame_records.FrameRecord(recipes["print"], w, h)
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=3))).cuda()
    outs = []
    with runtime.Owner() as owner:
        for _ in range(3):
            d = torch.zeros_like(src)
            owner.render(rec, src, d)
            outs.append(d.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])


def test_unsupported_stages_and_partial_windows_are_rejected(torch_cuda, recipes, prepare):
    from film_juicer_b200 import abi, frame_records, runtime

    torch = torch_cuda
    w, h = 32, 24
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(w, h, seed=3))).cuda()
    d = torch.zeros_like(src)
    rec = frame_records.FrameRecord(recipes["print"], w, h, grain=False, spatial_dir=False)
    with runtime.Owner() as owner:
        with pytest.raises(runtime.FjError, match="complete frame"):
            owner.render(rec, src, d, window=(2, 2, w, h))
        direct = frame_records.FrameRecord(recipes["direct"], w, h, grain=False, spatial_dir=False)
        direct.host.h.optics.flags |= abi.FJ_OPTICS_ENLARGER_DIFFUSION
        with pytest.raises(runtime.FjError, match="enlarger diffusion needs a print route") as e:
            owner.render(direct, src, d)
        assert e.value.status.category == abi.FJ_STATUS_UNSUPPORTED_INPUT
        rec.host.h.scanner_post.flags = 6  # unknown post-effect flags
        rec.host.h.scanner_post.hash = 1
        with pytest.raises(runtime.FjError, match="post effects"):
            owner.render(rec, src, d)
        rec.host.h.scanner_post.flags = 0
        rec.host.h.scanner_post.hash = 0
        rec.host.h.effects.flags |= abi.FJ_EFFECTS_FILM  # an active effects record without its identity
        with pytest.raises(runtime.FjError, match="identity"):
            owner.render(rec, src, d)
        rec.host.h.effects.flags = 0
