"""Fitting through spatial DIR (the development subtracts spatially filtered donor
corrections; fitting.FrameFit over fjb_fit_dir_source_carrier, the prepared DIR filter
(fjb_spatial_dir_filter_*), fjb_fit_forward_spatial_carrier / fjb_fit_vjp_spatial_carrier
and fjb_fit_dir_source_vjp_carrier):

* the DIR filter is symmetric, <G a, b> = <a, G b> within FP32 rounding, which makes
  it its own adjoint (half-sample reflected boundaries and symmetric components), and
  the prepared filter equals the one-shot fjb_spatial_dir_blur bit for bit;
* at the recipe's parameters the fitting source stage's filtered corrections equal the
  library's spatial-DIR stage (fjb_spatial_dir_build) on the same carrier;
* the 13 per-pixel parameters' gradient and the carrier-gradient planes equal autograd
  of the FP64 transcription (oracle/fit.py, with the library's filter as a linear map
  whose adjoint is itself) within 1e-3 relative, and the forward agrees with it, for a
  negative stock on the print route and for a positive stock (receiver Langmuir after
  the filter) scanned directly;
* L-BFGS through the frame Function recovers perturbed exposure and donor knees from a
  target render with spatial DIR and scatter/halation on."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
W, H = 160, 112


def _frame(torch, recipes, prepare, halation=False, seed=20261215, recipe="print"):
    from film_juicer_b200 import fitting, frame_records, runtime

    rec = frame_records.FrameRecord(recipes[recipe], W, H, recipe_hash=0x2101, diffusion=False, halation=halation,
                                    spatial_dir=True, grain=False, descriptor_width=W * 8)
    assert rec.host.h.spatial_dir.component_count > 0
    dr = runtime.DeviceRecipe(rec.host)
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=seed))).cuda()
    return rec, dr, src, fitting.FrameFit(dr, rec.host.h, src)


def _e0(torch, rec, carrier_rgb):
    route = float(rec.host.h.film_exposure.route_correction_scale)
    r, g, b = [p.double().reshape(-1) for p in carrier_rgb]
    return torch.clamp(torch.stack([b, g, r]) * route, min=0.0)


def _filter_fn(torch, ff):
    class Filter(torch.autograd.Function):
        """The library's DIR filter on (3, N) corrections (B, G, R receivers = Y, M, C
        planes); its adjoint is the same filter."""

        @staticmethod
        def forward(ctx, corr):
            out = ff.dir_filter([corr[j].detach().reshape(H, W).float().contiguous() for j in range(3)])
            return torch.stack([o.reshape(-1).double() for o in out])

        @staticmethod
        def backward(ctx, g):
            out = ff.dir_filter([g[j].reshape(H, W).float().contiguous() for j in range(3)])
            return torch.stack([o.reshape(-1).double() for o in out])

    return Filter.apply


def test_dir_filter_is_symmetric(torch_cuda, recipes, prepare):
    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare)
    gen = torch.Generator(device="cuda").manual_seed(5)
    a = [torch.randn((H, W), device="cuda", generator=gen) for _ in range(3)]
    b = [torch.randn((H, W), device="cuda", generator=gen) for _ in range(3)]
    ga, gb = ff.dir_filter(a), ff.dir_filter(b)
    # the prepared filter (fjb_spatial_dir_filter_apply) equals the one-shot entry
    from film_juicer_b200 import runtime

    once = [torch.empty_like(p) for p in a]
    runtime.spatial_dir_blur(rec.host.h.spatial_dir, a, once)
    for x, y in zip(ga, once):
        assert torch.equal(x, y)
    for c in range(3):
        lhs = float((ga[c].double() * b[c].double()).sum())
        rhs = float((a[c].double() * gb[c].double()).sum())
        scale = float(ga[c].double().norm() * b[c].double().norm())
        assert abs(lhs - rhs) <= 1e-5 * scale, (c, lhs, rhs)
        # the filter does something: it is not the identity
        assert float((ga[c] - a[c]).abs().max()) > 1e-3
    ff.close()
    dr.close()


def test_source_stage_equals_library_spatial_dir(torch_cuda, recipes, prepare):
    from film_juicer_b200 import fitting

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare)
    x0 = ff.x0
    th = fitting.default_theta(dr)
    ours = ff.filtered_corrections(th, x0)
    filtered = [torch.empty((H, W), device="cuda") for _ in range(3)]
    log_raw = [torch.empty((H, W), device="cuda") for _ in range(3)]
    dr.spatial_dir_build(rec.host.h.spatial_dir, filtered, log_raw, carrier=(x0[2], x0[1], x0[0]))
    torch.cuda.synchronize()
    for a, b in zip(ours, filtered):
        assert torch.all(torch.isfinite(a))
        assert float((a - b).abs().max()) <= 2e-6 * max(1.0, float(b.abs().max()))
    dr.close()


@pytest.mark.parametrize("recipe", ["print", "positive"])
def test_spatial_gradient_against_fp64_autograd(torch_cuda, recipes, prepare, recipe):
    from oracle import fit

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare, recipe=recipe)
    tab = fit.tables(rec.host)
    thp = torch.from_numpy(fit.perturbed_theta(tab))
    x = ff.x0
    gen = torch.Generator(device="cuda").manual_seed(7)
    w = torch.randn((3, H, W), device="cuda", generator=gen)
    g_theta, g_carrier = ff.vjp_carrier(thp, x, w)
    rgb = ff.forward(thp, ff.optics_default())
    ch = fit.Chain(torch, rec.host, device="cuda")
    carrier = [p.double().clone().requires_grad_(True) for p in x]
    th = thp.clone().cuda().requires_grad_(True)
    out = ch(_e0(torch, rec, carrier), th, spatial=_filter_fn(torch, ff))
    ref = out.detach().reshape(3, H, W)
    err = (rgb.double() - ref).abs()
    assert float((err - (2e-5 + 2e-4 * ref.abs())).max()) <= 0.0, float(err.max())
    (out * w.reshape(3, -1).double()).sum().backward()
    got, want = g_theta.cpu().numpy(), th.grad.cpu().numpy()
    used = fit.used_parameters(tab)
    assert np.linalg.norm(got[used] - want[used]) <= 1e-3 * np.linalg.norm(want[used]), (got, want)
    # the donor knees act through the filter: their gradient is not the runtime-DIR one
    # (positive stocks have no donor knees: theirs is zero)
    g_runtime, _ = fitting_vjp_runtime(torch, dr, thp, x, w)
    if recipe == "print":
        assert np.linalg.norm(got[9:12] - g_runtime[9:12]) > 1e-3 * np.linalg.norm(got[9:12])
    else:
        assert np.all(got[9:12] == 0.0)
    for gp, cp in zip(g_carrier, carrier):
        refg = cp.grad.reshape(H, W)
        assert float((gp.double() - refg).norm()) <= 1e-3 * float(refg.norm())
    dr.close()


def fitting_vjp_runtime(torch, dr, theta, carrier, w):
    from film_juicer_b200 import fitting

    g, gc = fitting.vjp_carrier(dr, theta, carrier, w)
    return g.cpu().numpy(), gc


def test_spatial_frame_fit_recovers_parameters(torch_cuda, recipes, prepare):
    from film_juicer_b200 import fitting

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare, halation=True)
    th0 = fitting.default_theta(dr).cpu()
    opt = ff.optics_default()
    truth = th0.clone()
    truth[0:3] += torch.tensor([0.12, -0.08, 0.05], dtype=truth.dtype)
    truth[9:12] *= torch.tensor([1.15, 0.9, 1.1], dtype=truth.dtype)
    target = ff.forward(truth, opt).clone()
    free = [0, 1, 2, 9, 10, 11]
    var = th0[free].clone().requires_grad_(True)
    lbfgs = torch.optim.LBFGS([var], lr=1.0, max_iter=80, line_search_fn="strong_wolfe")
    losses = []

    def closure():
        lbfgs.zero_grad()
        th = th0.index_put((torch.tensor(free),), var)
        rgb = fitting.frame_chain(th, opt, ff)
        loss = ((rgb - target) ** 2).mean() * 1e6
        loss.backward()
        losses.append(float(loss))
        return loss

    lbfgs.step(closure)
    assert losses[-1] <= 1e-4 * losses[0], (losses[0], losses[-1])
    got = var.detach()
    assert float((got[:3] - truth[:3]).abs().max()) <= 2e-3, (got, truth)
    assert float(((got[3:] - truth[9:12]) / truth[9:12]).abs().max()) <= 1e-2, (got, truth)
    dr.close()
