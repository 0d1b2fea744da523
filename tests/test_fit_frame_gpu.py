"""Fitting on whole frames with camera diffusion and scatter/halation on
(fitting.FrameFit over fjb_fit_forward_carrier / fjb_fit_vjp_carrier and the library's
diffusion and scatter/halation stages):

* the carrier that FrameFit forms (diffusion, then the scatter pass and the
  back-reflection pass run separately) is bit-identical to the full scatter/halation
  stage on the diffused carrier, and both optics stages are linear (Hal(x + t) =
  Hal(x) + Hal(t) within FP32 rounding), which the gradients of the optics
  parameters rely on;
* the carrier-input forward at the recipe's parameters with the optics off equals the
  source-input forward (the same exposure, rounded once more);
* the 13 per-pixel parameters' gradient and the carrier-gradient planes equal autograd
  of the FP64 transcription (oracle/fit.py) fed the library's carrier, within 1e-3
  relative;
* the optics tangents equal central differences of the library's carrier, and the
  optics parameters' gradient (camera scatter fraction, scatter amount, halation
  strength per channel) equals central differences (h = 1e-3) of the FP64
  transcription on the library's carrier within 2e-3 relative (a channel the record
  gives no back-reflection is not a free parameter);
* L-BFGS through the frame Function recovers perturbed scatter amount and halation
  strengths from a target render."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
W, H = 192, 128


def _frame(torch, recipes, prepare, diffusion=True, halation=True, seed=20261214):
    from film_juicer_b200 import fitting, frame_records, runtime

    rec = frame_records.FrameRecord(recipes["print"], W, H, recipe_hash=0x2001, diffusion=diffusion,
                                    halation=halation, spatial_dir=False, grain=False, descriptor_width=W * 8)
    dr = runtime.DeviceRecipe(rec.host)
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=seed))).cuda()
    return rec, dr, src, fitting.FrameFit(dr, rec.host.h, src)


def _e0(torch, rec, carrier_rgb):
    """FP64 film exposure B, G, R (3, N) as the capture stage forms it from the carrier."""
    route = float(rec.host.h.film_exposure.route_correction_scale)
    r, g, b = [p.double().reshape(-1) for p in carrier_rgb]
    return torch.clamp(torch.stack([b, g, r]) * route, min=0.0)


def test_stage_decomposition_and_linearity(torch_cuda, recipes, prepare):
    from film_juicer_b200 import runtime

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare)
    opt = ff.optics_default()
    x1, x2, x3 = ff.carriers(opt)
    full = [p.clone() for p in x1]
    runtime.scatter_halation(rec.host.h.optics.scatter_halation, full)
    for a, b in zip(full, x3):
        assert torch.equal(a, b)
    # linearity of both stages on a signed tangent-like plane
    t = [torch.randn_like(p) * 0.05 for p in x1]
    s = [p + q for p, q in zip(x1, t)]
    hs, hx, ht = [p.clone() for p in s], [p.clone() for p in x1], [p.clone() for p in t]
    for planes in (hs, hx, ht):
        runtime.scatter_halation(rec.host.h.optics.scatter_halation, planes)
    for a, b, c in zip(hs, hx, ht):
        err = float((a - b - c).abs().max())
        assert err <= 1e-5 * float(a.abs().max()), err
    ds, dx, dt = ff._diffuse(s, opt[0]), ff._diffuse(x1, opt[0]), ff._diffuse(t, opt[0])
    for a, b, c in zip(ds, dx, dt):
        err = float((a - b - c).abs().max())
        assert err <= 1e-5 * float(a.abs().max()), err
    dr.close()


def test_carrier_forward_equals_source_forward(torch_cuda, recipes, prepare):
    from film_juicer_b200 import fitting

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare, diffusion=False, halation=False)
    th = fitting.default_theta(dr)
    a = fitting.forward(dr, th, src)
    b = fitting.forward_carrier(dr, th, ff.x0)
    assert torch.all(torch.isfinite(b))
    err = (a - b).abs()
    assert float((err - (1e-5 + 1e-5 * a.abs())).max()) <= 0.0, float(err.max())
    dr.close()


def test_theta_gradient_and_carrier_planes(torch_cuda, recipes, prepare):
    from film_juicer_b200 import fitting
    from oracle import fit

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare)
    tab = fit.tables(rec.host)
    thp = torch.from_numpy(fit.perturbed_theta(tab))
    _, _, x3 = ff.carriers(ff.optics_default())
    w = torch.randn((3, H, W), device="cuda")
    g_theta, g_carrier = fitting.vjp_carrier(dr, thp, x3, w)
    ch = fit.Chain(torch, rec.host, device="cuda")
    carrier = [p.double().clone().requires_grad_(True) for p in x3]
    th = thp.clone().cuda().requires_grad_(True)
    out = ch(_e0(torch, rec, carrier), th)
    (out * w.reshape(3, -1).double()).sum().backward()
    got, want = g_theta.cpu().numpy(), th.grad.cpu().numpy()
    used = fit.used_parameters(tab)
    assert np.linalg.norm(got[used] - want[used]) <= 1e-3 * np.linalg.norm(want[used]), (got, want)
    for gp, cp in zip(g_carrier, carrier):
        ref = cp.grad.reshape(H, W)
        assert float((gp.double() - ref).norm()) <= 1e-3 * float(ref.norm())
    dr.close()


def test_optics_gradient_matches_central_differences(torch_cuda, recipes, prepare):
    from oracle import fit

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare)
    tab = fit.tables(rec.host)
    thp = torch.from_numpy(fit.perturbed_theta(tab))
    opt = ff.optics_default()
    # a mostly positive cotangent: with zero-mean weights the optics gradients are small
    # net sums of cancelling terms, and the difference quotients measure FP32 rounding
    gen = torch.Generator(device="cuda").manual_seed(3)
    w = 1.0 + 0.25 * torch.randn((3, H, W), device="cuda", generator=gen)
    g_theta, g_opt = ff.vjp(thp, opt, w)
    # tangents against central differences of the library's carrier
    x1, x2, x3 = ff.carriers(opt)
    tangents = ff.tangents(opt, x1, x2)
    # the record gives the blue channel no back-reflection (strength 0): not free
    assert tangents[4] is None and float(g_opt[4]) == 0.0
    for i in range(4):
        # the carrier is linear in f and a (and smooth in s): a wide step keeps the FP32
        # carriers' rounding out of the quotient
        h = 1e-2
        op, om = opt.clone(), opt.clone()
        op[i] += h
        om[i] -= h
        fd = [(a - b) / (2 * h) for a, b in zip(ff.carriers(op)[2], ff.carriers(om)[2])]
        num = sum(float((a.double() - b.double()).norm() ** 2) for a, b in zip(tangents[i], fd)) ** 0.5
        den = sum(float(b.double().norm() ** 2) for b in fd) ** 0.5
        assert num <= 1e-3 * den, (i, num, den)
    # the gradient against central differences of the FP64 chain on the library's carrier
    ch = fit.Chain(torch, rec.host, device="cuda")
    w64 = w.reshape(3, -1).double()
    th = thp.cuda()

    def loss(o):
        return float((ch(_e0(torch, rec, ff.carriers(o)[2]), th) * w64).sum())

    fd = np.zeros(5)
    for i in range(4):
        h = 1e-3
        op, om = opt.clone(), opt.clone()
        op[i] += h
        om[i] -= h
        fd[i] = (loss(op) - loss(om)) / (2 * h)
    got = g_opt.numpy()
    scale = np.abs(fd).max()
    for i in range(4):
        assert abs(got[i] - fd[i]) <= 2e-3 * abs(fd[i]) + 1e-4 * scale, (i, got, fd)
    dr.close()


def test_frame_fit_recovers_optics(torch_cuda, recipes, prepare):
    from film_juicer_b200 import fitting

    torch = torch_cuda
    rec, dr, src, ff = _frame(torch, recipes, prepare)
    th = fitting.default_theta(dr)
    opt0 = ff.optics_default()
    truth = opt0.clone()
    truth[1] *= 0.8   # scatter amount
    truth[2] += 0.05  # halation strength R
    truth[3] += 0.04  # halation strength G
    target = ff.forward(th, truth).clone()
    free = [1, 2, 3]
    var = opt0[free].clone().requires_grad_(True)
    lbfgs = torch.optim.LBFGS([var], lr=1.0, max_iter=60, line_search_fn="strong_wolfe")
    losses = []

    def closure():
        lbfgs.zero_grad()
        o = opt0.index_put((torch.tensor(free),), var)
        rgb = fitting.frame_chain(th, o, ff)
        loss = ((rgb - target) ** 2).mean() * 1e6  # a well-scaled objective for the line search
        loss.backward()
        losses.append(float(loss))
        return loss

    lbfgs.step(closure)
    assert losses[-1] <= 1e-4 * losses[0], (losses[0], losses[-1])
    assert float((var.detach() - truth[free]).abs().max()) <= 2e-3, (var, truth)
    dr.close()


def test_auto_exposure_frame_meters_once(torch_cuda, recipes, prepare):
    """With auto exposure on, FrameFit meters the source once (fjb_auto_exposure): its
    carrier is the unmetered carrier times the metered scale, and the parameters'
    gradient on it still equals FP64 autograd of the transcription."""
    from film_juicer_b200 import fitting, frame_records, runtime
    from oracle import fit

    torch = torch_cuda
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=20261216))).cuda()
    plain = frame_records.FrameRecord(recipes["print"], W, H, recipe_hash=0x2002, diffusion=False, halation=True,
                                      spatial_dir=False, grain=False, descriptor_width=W * 8)
    metered = frame_records.FrameRecord(recipes["print"], W, H, recipe_hash=0x2003, diffusion=False, halation=True,
                                        spatial_dir=False, grain=False, descriptor_width=W * 8, auto_exposure=True)
    dp, dm = runtime.DeviceRecipe(plain.host), runtime.DeviceRecipe(metered.host)
    fp, fm = fitting.FrameFit(dp, plain.host.h, src), fitting.FrameFit(dm, metered.host.h, src)
    scale = float(fm.meter_scale.cpu())
    assert np.isfinite(scale) and abs(scale - 1.0) > 1e-3
    for a, b in zip(fm.x0, fp.x0):
        err = (a.double() - b.double() * scale).abs()
        assert float((err - 4e-7 * (b.double() * scale).abs()).max()) <= 1e-30
    tab = fit.tables(metered.host)
    thp = torch.from_numpy(fit.perturbed_theta(tab))
    gen = torch.Generator(device="cuda").manual_seed(11)
    w = 1.0 + 0.25 * torch.randn((3, H, W), device="cuda", generator=gen)
    g_theta, g_opt = fm.vjp(thp, fm.optics_default(), w)
    _, _, x3 = fm.carriers(fm.optics_default())
    ch = fit.Chain(torch, metered.host, device="cuda")
    th = thp.clone().cuda().requires_grad_(True)
    (ch(_e0(torch, metered, x3), th) * w.reshape(3, -1).double()).sum().backward()
    used = fit.used_parameters(tab)
    got, want = g_theta.numpy(), th.grad.cpu().numpy()
    assert np.linalg.norm(got[used] - want[used]) <= 1e-3 * np.linalg.norm(want[used]), (got, want)
    dp.close()
    dm.close()


def test_highlight_reconstruction_frame(torch_cuda, recipes, prepare):
    """With highlight reconstruction on, FrameFit's carrier is the camera exposure after
    the reconstruction (fjb_highlight_boost on the camera exposure, applied once),
    and the parameters' gradient on the post-optics carrier equals FP64 autograd."""
    from film_juicer_b200 import descriptors, fitting, frame_records, runtime
    from oracle import fit

    torch = torch_cuda
    src = torch.from_numpy(np.ascontiguousarray(prepare.synthetic_frame(W, H, seed=20261217))).cuda()
    boost = descriptors.highlight_boost_record(protection=0.5, peak_gain=2.0)
    rec = frame_records.FrameRecord(recipes["print"], W, H, recipe_hash=0x2004, diffusion=True, halation=True,
                                    spatial_dir=False, grain=False, descriptor_width=W * 8, highlight_boost=boost)
    dr = runtime.DeviceRecipe(rec.host)
    ff = fitting.FrameFit(dr, rec.host.h, src)
    planes = [torch.empty((H, W), device="cuda") for _ in range(3)]
    dr.camera_exposure(src, planes)
    assert runtime.highlight_boost(boost, planes) == 1
    for a, b in zip(ff.x0, (planes[2], planes[1], planes[0])):
        assert torch.equal(a, b)
    tab = fit.tables(rec.host)
    thp = torch.from_numpy(fit.perturbed_theta(tab))
    gen = torch.Generator(device="cuda").manual_seed(12)
    w = 1.0 + 0.25 * torch.randn((3, H, W), device="cuda", generator=gen)
    g_theta, _ = ff.vjp(thp, ff.optics_default(), w)
    _, _, x3 = ff.carriers(ff.optics_default())
    ch = fit.Chain(torch, rec.host, device="cuda")
    th = thp.clone().cuda().requires_grad_(True)
    (ch(_e0(torch, rec, x3), th) * w.reshape(3, -1).double()).sum().backward()
    used = fit.used_parameters(tab)
    got, want = g_theta.numpy(), th.grad.cpu().numpy()
    assert np.linalg.norm(got[used] - want[used]) <= 1e-3 * np.linalg.norm(want[used]), (got, want)
    dr.close()
