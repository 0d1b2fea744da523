"""The fitting entry points (fjb_fit_defaults, fjb_fit_forward, fjb_fit_vjp) and the
torch.autograd.Function harness over them, against the oracle:

* the default parameters are the recipe's (the oracle's packed tables);
* the forward chain at the recipe's parameters equals the oracle's render to linear
  output RGB, and at a perturbed point the FP64 transcription (oracle/fit.py), within
  2e-4 + 3e-4 |rgb| (the render's processor bound);
* the hand-written adjoint on the differentiation workload (16 seeded 512 x 512 crops,
  one tall image) equals autograd of the FP64 transcription within 1e-3 relative
  (gradient-vector norm; per parameter 1e-3 |g| + 1e-4 max |g|), on the negative
  stock's direct and print routes, a positive stock scanned directly (receiver-Langmuir
  DIR) and the direct recipe with the Mallett 2019 reconstruction;
* it equals FP64 central differences (h = 1e-6) within the same bound, and the
  central differences (h = 1e-3) of the library's own FP32 forward within 2e-2 of the
  norm (a step of 1e-3 crosses the piecewise-linear curves' knots; the FP64 checks
  measure the function's exact derivative);
* the autograd.Function's backward is the adjoint, and Adam on it recovers perturbed
  exposure, gamma and print-exposure parameters from a target render;
* invalid parameters are rejected before any launch, and so is spatial DIR on a recipe
  without DIR couplers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _record(prepare, recipes, route):
    """The host record of a test route; "mallett" is the direct recipe with the Mallett
    2019 spectral reconstruction in place of the TC LUT."""
    from film_juicer_b200 import abi

    if route == "mallett":
        return prepare.HostRecord(recipes["direct"], method=abi.FJ_RAW_MALLETT_2019)
    return prepare.HostRecord(recipes[route])
BOUND = 1e-3


def _crops(prepare, n, size, seed):
    return np.ascontiguousarray(np.concatenate(
        [prepare.synthetic_frame(size, size, seed=seed + i) for i in range(n)], axis=0))


def _grad_close(got, want, used, bound=BOUND):
    got, want = np.asarray(got)[used], np.asarray(want)[used]
    assert np.linalg.norm(got - want) <= bound * np.linalg.norm(want), (got, want)
    scale = np.abs(want).max()
    for g, w in zip(got, want):
        assert abs(g - w) <= bound * abs(w) + 1e-4 * scale, (got, want)


@pytest.mark.parametrize("route", ["direct", "print", "positive", "mallett"])
def test_defaults_and_forward(torch_cuda, recipes, prepare, oracle, route):
    from film_juicer_b200 import fitting, runtime
    from oracle import fit

    torch = torch_cuda
    rec = _record(prepare, recipes, route)
    dr = runtime.DeviceRecipe(rec)
    tab = fit.tables(rec)
    th0 = fitting.default_theta(dr)
    assert np.array_equal(th0.numpy(), fit.default_theta(tab).astype(np.float32).astype(np.float64))
    src = np.ascontiguousarray(prepare.synthetic_frame(256, 160, seed=20261206))
    s = torch.from_numpy(src).cuda()
    got = fitting.forward(dr, th0, s).cpu().numpy()
    want = fit.linear_rgb(rec, src)
    assert np.all(np.isfinite(got))
    assert np.all(np.abs(got - want) <= 2e-4 + 3e-4 * np.abs(want)), float(np.abs(got - want).max())
    thp = fit.perturbed_theta(tab)
    got = fitting.forward(dr, torch.from_numpy(thp), s).cpu().numpy()
    ch = fit.Chain(torch, rec, device="cuda")
    e0 = torch.from_numpy(fit.exposure(rec, src).reshape(3, -1).astype(np.float64)).cuda()
    want = ch(e0, torch.from_numpy(thp).cuda()).cpu().numpy().reshape(got.shape)
    assert np.all(np.abs(got - want) <= 2e-4 + 3e-4 * np.abs(want)), float(np.abs(got - want).max())
    assert float(np.abs(got - fit.linear_rgb(rec, src)).max()) > 1e-3  # the parameters took effect
    dr.close()


@pytest.mark.parametrize("route", ["direct", "print", "positive", "mallett"])
def test_adjoint_matches_fp64_autograd_on_crop_batch(torch_cuda, recipes, prepare, oracle, route):
    """16 seeded 512 x 512 crops; the cotangent is the gradient of the mean squared
    error against a target rendered at the recipe's own parameters."""
    from film_juicer_b200 import fitting, runtime
    from oracle import fit

    torch = torch_cuda
    rec = _record(prepare, recipes, route)
    dr = runtime.DeviceRecipe(rec)
    tab = fit.tables(rec)
    src = _crops(prepare, 16, 512, 20261207)
    s = torch.from_numpy(src).cuda()
    thp = torch.from_numpy(fit.perturbed_theta(tab))
    ch = fit.Chain(torch, rec, device="cuda")
    e0 = torch.from_numpy(fit.exposure(rec, src).reshape(3, -1).astype(np.float64)).cuda()
    target = ch(e0, torch.from_numpy(fit.default_theta(tab)).cuda()).detach()
    th = thp.clone().cuda().requires_grad_(True)
    out = ch(e0, th)
    loss = ((out - target) ** 2).sum() / out.numel()
    loss.backward()
    want = th.grad.cpu().numpy()
    cot = (2.0 * (out.detach() - target) / out.numel()).to(torch.float32).reshape(3, *src.shape[:2]).contiguous()
    got = fitting.vjp(dr, thp, s, cot).cpu().numpy()
    used = fit.used_parameters(tab)
    assert np.all(got[[i for i in range(13) if i not in used]] == 0.0)
    _grad_close(got, want, used)
    # deterministic: a second call gives the same words
    again = fitting.vjp(dr, thp, s, cot).cpu().numpy()
    assert np.array_equal(got, again)
    dr.close()


@pytest.mark.parametrize("route", ["direct", "print", "positive", "mallett"])
def test_adjoint_matches_central_differences(torch_cuda, recipes, prepare, oracle, route):
    from film_juicer_b200 import fitting, runtime
    from oracle import fit

    torch = torch_cuda
    rec = _record(prepare, recipes, route)
    dr = runtime.DeviceRecipe(rec)
    tab = fit.tables(rec)
    src = np.ascontiguousarray(prepare.synthetic_frame(192, 128, seed=20261208))
    s = torch.from_numpy(src).cuda()
    thp = fit.perturbed_theta(tab)
    rng = np.random.default_rng(5)
    w = rng.standard_normal((3, 128, 192)).astype(np.float32)
    wt = torch.from_numpy(w).cuda()
    got = fitting.vjp(dr, torch.from_numpy(thp), s, wt).cpu().numpy()
    used = fit.used_parameters(tab)
    ch = fit.Chain(torch, rec, device="cuda")
    e0 = torch.from_numpy(fit.exposure(rec, src).reshape(3, -1).astype(np.float64)).cuda()
    w64 = wt.reshape(3, -1).double()

    def fd64(i, h):
        tp, tm = thp.copy(), thp.copy()
        tp[i] += h
        tm[i] -= h
        fp = ch(e0, torch.from_numpy(tp).cuda())
        fm = ch(e0, torch.from_numpy(tm).cuda())
        return float(((fp - fm) * w64).sum()) / (2 * h)

    _grad_close(got, [fd64(i, 1e-6) if i in used else 0.0 for i in range(13)], used)

    def fd32(i, h):
        tp, tm = thp.copy(), thp.copy()
        tp[i] += h
        tm[i] -= h
        fp = fitting.forward(dr, torch.from_numpy(tp), s).double()
        fm = fitting.forward(dr, torch.from_numpy(tm), s).double()
        return float(((fp - fm) * wt.double()).sum()) / (2 * h)

    fd = np.array([fd32(i, 1e-3) if i in used else 0.0 for i in range(13)])
    assert np.linalg.norm(got[used] - fd[used]) <= 2e-2 * np.linalg.norm(fd[used]), (got, fd)
    dr.close()


@pytest.mark.parametrize("side", ["camera", "print"])
def test_autograd_function_and_fit(torch_cuda, recipes, prepare, oracle, side):
    """Adam through the Function recovers the parameters a target was rendered with:
    the camera side (exposure and film gamma per layer) or the print side (print gamma
    per dye and print exposure). The common part of the three camera exposures and the
    print exposure move the print's exposure alike, so one side is fitted at a time."""
    from film_juicer_b200 import fitting, runtime

    torch = torch_cuda
    rec = prepare.HostRecord(recipes["print"])
    dr = runtime.DeviceRecipe(rec)
    src = torch.from_numpy(_crops(prepare, 4, 128, 20261209)).cuda()
    th0 = fitting.default_theta(dr)
    truth = th0.clone()
    if side == "camera":
        free = [0, 1, 2, 3, 4, 5]
        truth[[0, 1, 2]] += torch.tensor([0.15, -0.1, 0.08], dtype=torch.float64)
        truth[[3, 4, 5]] *= torch.tensor([1.04, 0.97, 1.02], dtype=torch.float64)
    else:
        free = [6, 7, 8, 12]
        truth[[6, 7, 8]] *= torch.tensor([0.96, 1.03, 1.05], dtype=torch.float64)
        truth[12] -= 0.12
    target = fitting.forward(dr, truth, src).clone()
    # backward of the Function is the adjoint
    th = th0.clone().requires_grad_(True)
    rgb = fitting.chain(th, dr, src)
    (rgb * target).sum().backward()
    direct = fitting.vjp(dr, th0, src, target).cpu()
    assert torch.equal(th.grad, direct)
    theta, losses = fitting.fit(dr, src, target, th0, free=free, steps=300, lr=0.01)
    assert losses[-1] <= 1e-4 * losses[0], (losses[0], losses[-1])
    assert float((theta[free] - truth[free]).abs().max()) <= 5e-3, (theta, truth)
    dr.close()


def test_unsupported_cases_are_rejected(torch_cuda, recipes, prepare):
    from film_juicer_b200 import abi, fitting, runtime

    torch = torch_cuda
    src = torch.zeros((8, 8, 3), device="cuda")
    g = torch.zeros((3, 8, 8), device="cuda")
    rec = prepare.HostRecord(recipes["direct"])
    dr = runtime.DeviceRecipe(rec)
    th = fitting.default_theta(dr)
    bad = th.clone()
    bad[9] = 0.0
    with pytest.raises(runtime.FjError) as e:
        fitting.forward(dr, bad, src)
    assert e.value.status.category == abi.FJ_STATUS_UNSUPPORTED_INPUT
    bad = th.clone()
    bad[0] = float("nan")
    with pytest.raises(runtime.FjError):
        fitting.vjp(dr, bad, src, g)
    dr.close()
    # a recipe without DIR couplers is still a valid fitting problem; spatial DIR on it is not
    rec = prepare.HostRecord(recipes["direct"])
    rec.h.dir_couplers.mode = abi.FJ_DIR_INACTIVE
    dr = runtime.DeviceRecipe(rec)
    planes = [torch.zeros((8, 8), device="cuda") for _ in range(3)]
    assert torch.all(torch.isfinite(fitting.forward(dr, fitting.default_theta(dr), src)))
    with pytest.raises(runtime.FjError) as e:
        fitting.dir_source_carrier(dr, fitting.default_theta(dr), planes)
    assert e.value.status.category == abi.FJ_STATUS_UNSUPPORTED_INPUT
    dr.close()
