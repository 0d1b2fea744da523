"""Auto-exposure metering (a14) on the GPU against the oracle.

The device reduction sums FP64 partials in a different order than the oracle's
sequential loop, so the metered mean agrees to ~1e-15 relative; the float scale is
required to agree to 2 ulp. Median metering is rejected like the reference
(src/Cuda/JuicerCudaExecutor.cpp:3145)."""
import numpy as np
import pytest

from film_juicer_b200 import abi

pytestmark = pytest.mark.gpu
METHODS = [abi.FJ_METER_CENTER_WEIGHTED, abi.FJ_METER_AVERAGE, 3, 4, 5, 6]


@pytest.fixture(scope="module")
def direct(torch_cuda, recipes, prepare):
    from film_juicer_b200 import runtime

    rec = prepare.HostRecord(recipes["direct"], auto_exposure=True)
    dr = runtime.DeviceRecipe(rec)
    yield rec, dr
    dr.close()


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("shape", [(640, 360), (333, 517), (2, 3)])
def test_meter_scale_matches_oracle(torch_cuda, direct, prepare, oracle, method, shape):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec, dr = direct
    w, h = shape
    src = prepare.synthetic_frame(w, h, seed=99 + method)
    meter = runtime.meter_record(w, h, method=method)
    s = torch.from_numpy(src).cuda()
    scale = torch.zeros(1, device="cuda")
    runtime.auto_exposure(dr, s, meter, scale)
    got = float(scale.item())
    ref = oracle.auto_exposure(rec, meter, src)
    assert ref is not None and np.isfinite(got) and got > 0
    ulp = abs(np.array([got], np.float32).view(np.int32)[0] - np.array([ref], np.float32).view(np.int32)[0])
    assert ulp <= 2, (got, ref)


def test_meter_is_deterministic_and_windowed(torch_cuda, direct, prepare, oracle):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec, dr = direct
    src = prepare.synthetic_frame(1024, 768, seed=5)
    s = torch.from_numpy(src).cuda()
    meter = runtime.meter_record(1024, 768, meter=(100, 50, 900, 700), preview=(200, 162))
    vals = []
    for _ in range(3):
        scale = torch.zeros(1, device="cuda")
        runtime.auto_exposure(dr, s, meter, scale)
        vals.append(float(scale.item()))
    assert vals[0] == vals[1] == vals[2]
    ref = oracle.auto_exposure(rec, meter, src)
    assert abs(vals[0] - ref) <= 4e-7 * ref


def test_median_metering_is_rejected(torch_cuda, direct, prepare):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    _, dr = direct
    s = torch.zeros((8, 8, 3), device="cuda")
    meter = runtime.meter_record(8, 8, method=abi.FJ_METER_MEDIAN)
    with pytest.raises(runtime.FjError) as e:
        runtime.auto_exposure(dr, s, meter, torch.zeros(1, device="cuda"))
    assert e.value.status.category == abi.FJ_STATUS_UNSUPPORTED_INPUT


def test_metered_scale_feeds_the_render(torch_cuda, direct, prepare, oracle):
    """The scale written by the meter is read by the exposure step of the render."""
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec, dr = direct
    src = prepare.synthetic_frame(160, 90, seed=3)
    s = torch.from_numpy(src).cuda()
    scale = torch.zeros(1, device="cuda")
    runtime.auto_exposure(dr, s, runtime.meter_record(160, 90), scale)
    dr.set_exposure_scale_device(scale)
    out = torch.empty_like(s)
    dr.render(s, out)
    dr.set_exposure_scale_device(None)
    ref, _ = oracle.render(rec, src, auto_scale=float(scale.item()))
    assert np.all(np.abs(out.cpu().numpy() - ref) <= 2e-4 + 3e-4 * np.abs(ref))


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("shape", [(640, 360), (333, 517), (1920, 1080), (2, 3)])
def test_meter_scale_matches_reference_cuda(torch_cuda, direct, prepare, oracle, method, shape):
    """The reference's own metering launchers (compiled from its sources into the
    harness) on the same frame and record: the float scale agrees to 1 ulp (both sum
    FP64 partials, in different orders)."""
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec, dr = direct
    w, h = shape
    src = prepare.synthetic_frame(w, h, seed=7 + method)
    meter = runtime.meter_record(w, h, method=method)
    ref = oracle.reference_auto_exposure(torch, rec, meter, src)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    scale = torch.zeros(1, device="cuda")
    runtime.auto_exposure(dr, torch.from_numpy(src).cuda(), meter, scale)
    got = float(scale.item())
    ulp = abs(np.array([got], np.float32).view(np.int32)[0] - np.array([ref], np.float32).view(np.int32)[0])
    assert ulp <= 1, (got, ref)


def test_windowed_meter_matches_reference_cuda(torch_cuda, direct, prepare, oracle):
    torch = torch_cuda
    from film_juicer_b200 import runtime

    rec, dr = direct
    src = prepare.synthetic_frame(1024, 768, seed=5)
    meter = runtime.meter_record(1024, 768, meter=(100, 50, 900, 700), preview=(200, 162))
    ref = oracle.reference_auto_exposure(torch, rec, meter, src)
    if ref is None:
        pytest.skip("reference CUDA harness not built")
    scale = torch.zeros(1, device="cuda")
    runtime.auto_exposure(dr, torch.from_numpy(src).cuda(), meter, scale)
    got = float(scale.item())
    assert abs(np.array([got], np.float32).view(np.int32)[0] - np.array([ref], np.float32).view(np.int32)[0]) <= 1
