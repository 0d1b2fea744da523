"""The FP64 transcription of the parameterised per-pixel chain (oracle/fit.py), the
checker of the library's fitting adjoint, checked on the CPU:

* at the recipe's parameters it reproduces the oracle's FP32 render to linear output
  RGB (oracle stage 7) within 2e-6 + 1e-5 |rgb|, on both golden recipes;
* the DIR compensated axes that it rebuilds from the donor knees equal the recipe's
  axes (the reference host's build, rust/film-juicer-core/src/film/dir.rs:258-290)
  within 4e-7, so a knee change moves the axes as the host would;
* its autograd gradient of a weighted sum of the output agrees with central finite
  differences in FP64: with h = 1e-6 within 1e-3 relative (of the gradient vector's
  norm, and per parameter 1e-3 |fd| + 1e-4 max |fd|); with h = 1e-3 within 1e-2 of the
  norm. The chain's curves are piecewise linear (sampled density curves, the scanner
  LUT's cells), so a step of 1e-3 moves many pixels across sample knots and its
  difference quotient averages the slopes on both sides: on these recipes it differs
  from the exact derivative by 0.3-0.5 % of the norm, a property of the function, not of
  the gradient.
"""
import numpy as np
import pytest



def _record(prepare, recipes, route):
    """The host record of a test route; "mallett" is the direct recipe with the Mallett
    2019 spectral reconstruction in place of the TC LUT."""
    from film_juicer_b200 import abi

    if route == "mallett":
        return prepare.HostRecord(recipes["direct"], method=abi.FJ_RAW_MALLETT_2019)
    return prepare.HostRecord(recipes[route])

@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


@pytest.mark.parametrize("route", ["direct", "print", "positive", "mallett"])
def test_transcription_matches_oracle_linear_render(torch, recipes, prepare, oracle, route):
    from oracle import fit

    rec = _record(prepare, recipes, route)
    ch = fit.Chain(torch, rec)
    src = np.ascontiguousarray(prepare.synthetic_frame(96, 64, seed=7))
    e0 = fit.exposure(rec, src)
    want = fit.linear_rgb(rec, src)
    theta = torch.tensor(fit.default_theta(ch.tab), dtype=torch.float64)
    got = ch(torch.from_numpy(e0.reshape(3, -1).astype(np.float64)), theta).numpy().reshape(want.shape)
    assert np.all(np.isfinite(got)) and np.all(np.isfinite(want))
    assert np.all(np.abs(got - want) <= 2e-6 + 1e-5 * np.abs(want)), float(np.abs(got - want).max())
    ax = ch.axes(torch.tensor(ch.tab["dir_k"])).numpy()
    assert float(np.abs(ax - ch.tab["axes_bgr"]).max()) <= 4e-7


def _fd_case(torch, fit, prepare, rec, seed):
    ch = fit.Chain(torch, rec)
    rng = np.random.default_rng(seed)
    src = np.ascontiguousarray(prepare.synthetic_frame(48, 32, seed=seed))
    e0 = torch.from_numpy(fit.exposure(rec, src).reshape(3, -1).astype(np.float64))
    theta0 = torch.from_numpy(fit.perturbed_theta(ch.tab))
    w = torch.from_numpy(rng.standard_normal((3, e0.shape[1])))
    return ch, e0, theta0, w


@pytest.mark.parametrize("route", ["direct", "print", "positive", "mallett"])
def test_transcription_gradient_matches_finite_differences(torch, recipes, prepare, oracle, route):
    from oracle import fit

    rec = _record(prepare, recipes, route)
    ch, e0, theta0, w = _fd_case(torch, fit, prepare, rec, 11)
    th = theta0.clone().requires_grad_(True)
    (ch(e0, th) * w).sum().backward()
    grad = th.grad.numpy()
    used = fit.used_parameters(ch.tab)
    unused = [i for i in range(13) if i not in used]
    assert np.all(grad[unused] == 0.0)
    for h, bound in ((1e-6, 1e-3), (1e-3, 1e-2)):
        fd = central_differences(ch, e0, theta0, w, h)
        assert np.all(fd[unused] == 0.0)
        assert np.linalg.norm(grad - fd) <= bound * np.linalg.norm(fd), (h, grad, fd)
        if h < 1e-4:
            scale = np.abs(fd).max()
            for i in used:
                assert abs(grad[i] - fd[i]) <= 1e-3 * abs(fd[i]) + 1e-4 * scale, (i, grad[i], fd[i])


def central_differences(ch, e0, theta0, w, h):
    fd = np.zeros(13)
    for i in range(13):
        tp, tm = theta0.clone(), theta0.clone()
        tp[i] += h
        tm[i] -= h
        fd[i] = float(((ch(e0, tp) - ch(e0, tm)) * w).sum()) / (2 * h)
    return fd
