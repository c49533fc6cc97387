"""GPU gradients: the adjoint kernels (gsb_adjoint_images through autodiff) against central
finite differences of the FP64 drawing path.

Nothing in the reference computes derivatives, so gradient parity rests on finite differences
of the forward path, whose own parity with the reference is pinned by test_gpu_parity.py.

* Record level (every leaf type, phases, scales): FP64 adjoint vs FP64 central differences of
  a random linear functional of the stamps, relative step 1e-6; agreement 1e-5 relative to the
  largest gradient entry of the same kind.
* Fit step (Sersic x Moffat(2.5, 0.8) x Pixel(0.2), 48x48, chi^2 at SNR 50), gradients in
  (flux, hlr, n, g1, g2, dx, dy) against FP64 central differences with step 1e-4, compared in
  natural units (d/dln flux, d/dln hlr, d/dn, d/dg1, d/dg2, d/d(dx / pixel), d/d(dy / pixel)):
  - the FP64 adjoint: every entry to 1e-5 of the stamp's largest entry;
  - the FP32 adjoint (FP32 kValue, k-product and FFT): norm-wise 1e-4 per stamp, i.e. the
    largest error is at most 1e-4 of the largest entry, and entries of at least 10% of the
    largest agree to 1e-4 relative.  Smaller entries (e.g. the centroid gradient of a nearly
    shift-invariant loss) carry the FP32 rounding of the others, and the FP32 chi^2 itself
    differs from the FP64 one through the FP32 image in its residual.
"""
import numpy as np
import pytest

import galsim_b200 as galsim
from galsim_b200 import autodiff

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def _trees():
    rng = np.random.default_rng(7)
    B = 3

    def u(a, b):
        return rng.uniform(a, b, B)

    pix = galsim.Pixel(0.2)
    yield 'sersic_hlr_moffat25', galsim.Convolve(
        galsim.Sersic(n=u(0.8, 3.5), half_light_radius=u(0.4, 0.9), flux=u(1e3, 5e3))
        .shear(g1=u(-0.2, 0.2), g2=u(-0.2, 0.2)).shift(u(-0.2, 0.2), u(-0.2, 0.2)),
        galsim.Moffat(beta=2.5, fwhm=0.8), pix)
    ns = u(1.0, 4.0)
    yield 'sersic_r0_kolmogorov', galsim.Convolve(
        galsim.Sersic(n=ns, scale_radius=u(0.4, 0.8) / (2. * ns - 1. / 3.) ** ns, flux=u(1e3, 5e3))
        .shear(g1=u(-0.2, 0.2), g2=u(-0.2, 0.2)),
        galsim.Kolmogorov(fwhm=u(0.6, 0.9)), pix)
    yield 'exp_gauss_sum_airy', galsim.Convolve(
        galsim.Add(galsim.Exponential(half_light_radius=u(0.5, 1.0), flux=u(500., 900.))
                   .shear(g1=u(-0.2, 0.2), g2=u(-0.2, 0.2)),
                   galsim.Gaussian(sigma=u(0.2, 0.4), flux=u(100., 300.)).shift(u(-0.3, 0.3), u(-0.3, 0.3))),
        galsim.Airy(lam_over_diam=0.12, obscuration=0.3), pix)
    yield 'moffat_modes_box_scale', galsim.Convolve(
        galsim.Moffat(beta=3.3, half_light_radius=u(0.4, 0.7), flux=u(1e3, 2e3)).shear(g1=u(-0.1, 0.1), g2=u(-0.1, 0.1)),
        galsim.Moffat(beta=1.5, scale_radius=0.3) * 1.7,
        galsim.Moffat(beta=3.5, fwhm=0.5),
        galsim.Box(0.3, 0.2))
    # the mixed bulge+disk configuration at its own GSParams: Sersic(n=4) + Exponential with
    # independent shears, general-beta Moffat, minimum_fft_size=32
    gsp = galsim.GSParams(minimum_fft_size=32)
    yield 'bulge_disk_moffat_gen_min32', galsim.Convolve(
        galsim.Add(galsim.Sersic(n=4., half_light_radius=u(0.3, 0.5), flux=u(1e3, 3e3), gsparams=gsp)
                   .shear(g1=u(-0.3, 0.3), g2=u(-0.3, 0.3)),
                   galsim.Exponential(half_light_radius=u(0.6, 1.0), flux=u(2e3, 5e3), gsparams=gsp)
                   .shear(g1=u(-0.3, 0.3), g2=u(-0.3, 0.3))),
        galsim.Moffat(beta=u(2.6, 4.4), fwhm=u(0.5, 1.0), gsparams=gsp), galsim.Pixel(0.2, gsparams=gsp))
    yield 'gauss_diag_airy_unobscured', galsim.Convolve(
        galsim.Gaussian(sigma=u(0.3, 0.5), flux=u(1e3, 2e3)).dilate(u(0.9, 1.2)),
        galsim.Airy(lam_over_diam=0.15), galsim.Kolmogorov(fwhm=0.7), pix)


def _loss(img, w):
    return float((img.double() * w).sum())


def _fd(plan, base, w, field, idx, h, sizes):
    vals = []
    for sgn in (1., -1.):
        rec = {k: v.clone() for k, v in base.items()}
        rec[field][idx] += sgn * h
        plan.set_records(rec)
        img = plan.draw()
        if not (np.array_equal(plan.last.N, sizes[0]) and np.array_equal(plan.last.Nk, sizes[1])):
            return None
        vals.append(_loss(img, w))
    return (vals[0] - vals[1]) / (2. * h)


@pytest.mark.parametrize('name,obj', list(_trees()), ids=[t[0] for t in _trees()])
def test_record_gradients_fp64_vs_finite_differences(name, obj):
    _check_record_gradients(name, obj, 40, 40, 0.2)


def _large_trees():
    """Trees drawn with FFT sizes above 1024 (the split large-FFT path and its adjoint)."""
    rng = np.random.default_rng(17)
    B = 2

    def u(a, b):
        return rng.uniform(a, b, B)

    g1536 = galsim.GSParams(minimum_fft_size=1536)
    yield 'sersic_airy_N1536', 1536, galsim.Convolve(
        galsim.Sersic(n=u(1.5, 3.5), half_light_radius=u(0.4, 0.7), flux=u(1e3, 5e3), gsparams=g1536)
        .shear(g1=u(-0.2, 0.2), g2=u(-0.2, 0.2)).shift(u(-0.1, 0.1), u(-0.1, 0.1)),
        galsim.Airy(lam_over_diam=0.1, obscuration=0.3, gsparams=g1536), galsim.Pixel(0.05, gsparams=g1536))
    g2048 = galsim.GSParams(minimum_fft_size=2048)
    yield 'exp_gauss_sum_moffat_N2048', 2048, galsim.Convolve(
        galsim.Add(galsim.Exponential(half_light_radius=u(0.3, 0.5), flux=u(500., 900.), gsparams=g2048)
                   .shear(g1=u(-0.2, 0.2), g2=u(-0.2, 0.2)),
                   galsim.Gaussian(sigma=u(0.1, 0.2), flux=u(100., 300.), gsparams=g2048)
                   .shift(u(-0.1, 0.1), u(-0.1, 0.1))),
        galsim.Moffat(beta=3.0, fwhm=0.4, gsparams=g2048), galsim.Pixel(0.05, gsparams=g2048))


@pytest.mark.parametrize('name,N,obj', list(_large_trees()), ids=[t[0] for t in _large_trees()])
def test_record_gradients_large_fft_fp64_vs_finite_differences(name, N, obj):
    """The adjoint of the split large-FFT path (N > 1024) against FP64 central differences."""
    plan = _check_record_gradients(name, obj, 64, 64, 0.05)
    assert np.all(plan.last.N == N)


@pytest.mark.parametrize('name,N,obj', list(_large_trees()), ids=[t[0] for t in _large_trees()])
def test_large_fft_adjoint_fp32_vs_fp64(name, N, obj):
    w = None
    grads = []
    for prec, dt in (('fp64', np.float64), ('fp32', np.float32)):
        plan = autodiff.RecordPlan(obj, 64, 64, 0.05, dtype=dt, precision=prec)
        base = plan.records()
        plan.set_records(base)
        img = plan.draw()
        assert np.all(plan.last.N == N)
        if w is None:
            w = np.random.default_rng(5).standard_normal(tuple(img.shape))
        grads.append(plan.adjoint(torch.as_tensor(w, device=img.device, dtype=img.dtype)))
    for field in autodiff.RECORD_FIELDS:
        a, b = grads[0][field].cpu().numpy(), grads[1][field].cpu().numpy()
        if a.size == 0:
            continue
        top = np.abs(a).max()
        assert np.abs(a - b).max() <= 1e-4 * max(top, 1e-30), (name, field, np.abs(a - b).max(), top)


def _check_record_gradients(name, obj, nx, ny, scale):
    plan = autodiff.RecordPlan(obj, nx, ny, scale, dtype=np.float64, precision='fp64')
    base = plan.records()
    plan.set_records(base)
    img = plan.draw()
    sizes = (plan.last.N.copy(), plan.last.Nk.copy())
    w = torch.as_tensor(np.random.default_rng(3).standard_normal(tuple(img.shape)), device=img.device)
    g = plan.adjoint(w)
    B = plan.B
    checked = 0
    for field in autodiff.RECORD_FIELDS:
        ga = g[field].cpu().numpy()
        if ga.size == 0:
            continue
        scale_ref = np.abs(ga).max()
        for idx in np.ndindex(*ga.shape[1:]):
            l = idx[0]
            if field == 'leaf_n' and plan.types[l] != galsim._lib.SERSIC:
                continue
            if field == 'leaf_size' and idx[1] == 1 and plan.types[l] != galsim._lib.BOX:
                continue
            for s in range(B):
                full = (s,) + idx
                v0 = float(base[field][full])
                if field in ('leaf_jac', 'phase_jac') and idx[1] in (1, 2):
                    # off-diagonal: only where the Jacobian is already general (the 1-d and 2-d
                    # fill rules clip differently)
                    jb = base[field][(s, l)]
                    if float(jb[1]) == 0. and float(jb[2]) == 0.:
                        continue
                h = 1e-6 * max(abs(v0), 1e-3 if field != 'phase_cen' else 1e-2)
                fd = _fd(plan, base, w, field, full, h, sizes)
                if fd is None:
                    continue
                err = abs(ga[full] - fd)
                assert err <= 1e-5 * max(abs(fd), 1e-2 * scale_ref), (name, field, full, ga[full], fd)
                checked += 1
    assert checked > 20
    return plan


def _fit_problem(B=6, seed=11):
    rng = np.random.default_rng(seed)
    flux = 1e4 * np.exp(rng.normal(0., 0.5, B))
    hlr = rng.uniform(0.3, 1.2, B)
    n = rng.uniform(1., 3., B)
    g1 = rng.normal(0., 0.1, B)
    g2 = rng.normal(0., 0.1, B)
    dx = rng.normal(0., 0.1, B)
    dy = rng.normal(0., 0.1, B)
    true = np.stack([flux, hlr, n, g1, g2, dx, dy], -1)
    pert = true * (1. + rng.normal(0., 0.03, true.shape)) + rng.normal(0., 0.02, true.shape) * \
        np.array([0., 0., 0., 1., 1., 1., 1.])
    return true, pert, rng


def _natural(g, p):
    """Gradient in natural units: relative for flux and hlr, per pixel (0.2") for dx, dy."""
    s = np.stack([p[:, 0], p[:, 1], np.ones(len(p)), np.ones(len(p)), np.ones(len(p)),
                  np.full(len(p), 0.2), np.full(len(p), 0.2)], -1)
    return g * s


def _assert_grad_close(g, ref, p, tol, big_frac=0.1):
    gn, rn = _natural(g, p), _natural(ref, p)
    top = np.abs(rn).max(axis=1, keepdims=True)
    err = np.abs(gn - rn)
    assert np.all(err <= tol * top), (err / top).max()
    big = np.abs(rn) >= big_frac * top
    assert np.all(err[big] <= tol * np.abs(rn[big])), (err[big] / np.abs(rn[big])).max()


def _chi2_problem(B, seed):
    psf = galsim.Convolve(galsim.Moffat(beta=2.5, fwhm=0.8), galsim.Pixel(0.2))
    true, pert, rng = _fit_problem(B, seed)
    dev = galsim._lib.Device.torch_device()
    m64 = autodiff.GalaxyModel(psf, 48, 48, 0.2, dtype=np.float64, precision='fp64')
    timg = m64(torch.as_tensor(true, device=dev)).detach()
    sigma = torch.sqrt((timg ** 2).sum(dim=(1, 2))) / 50.
    target = timg + sigma[:, None, None] * torch.as_tensor(rng.standard_normal(tuple(timg.shape)), device=dev)

    def chi2_per_stamp(img):
        return (((img.double() - target) / sigma[:, None, None]) ** 2).sum(dim=(1, 2))

    def adjoint_grad(model):
        p = torch.as_tensor(pert, device=dev, dtype=torch.float64).requires_grad_(True)
        chi2_per_stamp(model(p)).sum().backward()
        return p.grad.cpu().numpy()

    def fd_grad():
        fd = np.zeros_like(pert)
        for j in range(7):
            h = 1e-4 * (pert[:, j] if j in (0, 1) else np.ones(len(pert)))
            for sgn in (1., -1.):
                q = pert.copy()
                q[:, j] += sgn * h
                with torch.no_grad():
                    per = chi2_per_stamp(m64(torch.as_tensor(q, device=dev)))
                fd[:, j] += sgn * per.cpu().numpy() / (2. * h)
        return fd

    return psf, pert, m64, adjoint_grad, fd_grad


def test_fit_step_gradient_fp64_adjoint_vs_fp64_finite_differences():
    psf, pert, m64, adjoint_grad, fd_grad = _chi2_problem(6, 11)
    _assert_grad_close(adjoint_grad(m64), fd_grad(), pert, 1e-5, big_frac=1.1)


def test_fit_step_gradient_fp32_adjoint_vs_fp64_finite_differences():
    psf, pert, m64, adjoint_grad, fd_grad = _chi2_problem(6, 11)
    m32 = autodiff.GalaxyModel(psf, 48, 48, 0.2, dtype=np.float32, precision='fp32')
    _assert_grad_close(adjoint_grad(m32), fd_grad(), pert, 1e-4)


def test_fit_step_fp64_adjoint_matches_fp32_adjoint():
    psf = galsim.Convolve(galsim.Moffat(beta=2.5, fwhm=0.8), galsim.Pixel(0.2))
    true, pert, rng = _fit_problem(B=4, seed=5)
    dev = galsim._lib.Device.torch_device()
    grads = []
    for prec, dt in (('fp32', np.float32), ('fp64', np.float64)):
        m = autodiff.GalaxyModel(psf, 48, 48, 0.2, dtype=dt, precision=prec)
        p = torch.as_tensor(pert, device=dev, dtype=torch.float64).requires_grad_(True)
        w = torch.as_tensor(np.random.default_rng(2).standard_normal((len(pert), 48, 48)), device=dev)
        (m(p).double() * w).sum().backward()
        grads.append(p.grad.cpu().numpy())
    _assert_grad_close(grads[0], grads[1], pert, 1e-4)


def test_adjoint_requires_dn_tables_for_sersic():
    obj = galsim.Convolve(galsim.Sersic(n=np.array([1.5, 2.5]), half_light_radius=0.5), galsim.Pixel(0.2))
    plan = autodiff.RecordPlan(obj, 32, 32, 0.2)
    plan.prog.need_dn = False
    img = plan.draw()
    with pytest.raises(galsim.GalSimError):
        plan.adjoint(torch.ones_like(img))


def test_backward_after_a_later_forward_with_shared_tables():
    """GalaxyModel reuses one device table set; a graph whose tables were rebuilt by a later
    forward call still gets its own gradients."""
    psf = galsim.Convolve(galsim.Moffat(beta=2.5, fwhm=0.8), galsim.Pixel(0.2))
    _, pert, _ = _fit_problem(B=3, seed=9)
    dev = galsim._lib.Device.torch_device()
    m = autodiff.GalaxyModel(psf, 48, 48, 0.2, dtype=np.float64, precision='fp64')
    w = torch.as_tensor(np.random.default_rng(4).standard_normal((3, 48, 48)), device=dev)
    p1 = torch.as_tensor(pert, device=dev).requires_grad_(True)
    (m(p1) * w).sum().backward()
    ref = p1.grad.clone()
    p1.grad = None
    loss1 = (m(p1) * w).sum()
    q = pert.copy()
    q[:, 2] += 0.7                      # different Sersic n: the shared tables are rebuilt
    m(torch.as_tensor(q, device=dev))
    loss1.backward()
    assert torch.allclose(p1.grad, ref, rtol=1e-12, atol=0.)


def test_want_mask_factored_sum_atom_matches_full_adjoint():
    """Gradients of the bulge and disk of Sum(Sersic, Exponential) (x Moffat x Pixel) computed
    with a want mask (factored pass; the Sum is one atom whose cotangent reaches both leaves)
    equal those of the full reverse pass over every record; unwanted entries are zero."""
    rng = np.random.default_rng(13)
    B = 4
    bulge = galsim.Sersic(n=4., half_light_radius=rng.uniform(0.3, 0.5, B), flux=rng.uniform(100., 300., B))
    disk = galsim.Exponential(half_light_radius=rng.uniform(0.6, 1.0, B), flux=rng.uniform(300., 700., B))
    obj = galsim.Convolve(galsim.Add(bulge.shear(g1=rng.uniform(-0.2, 0.2, B), g2=rng.uniform(-0.2, 0.2, B)),
                                     disk.shear(g1=rng.uniform(-0.2, 0.2, B), g2=rng.uniform(-0.2, 0.2, B))),
                          galsim.Moffat(beta=3.7, fwhm=0.7), galsim.Pixel(0.2))
    for prec, dt, tol in (('fp64', np.float64, 1e-9), ('fp32', np.float32, 2e-5)):
        plan = autodiff.RecordPlan(obj, 48, 48, 0.2, dtype=dt, precision=prec)
        img = plan.draw()
        w = torch.as_tensor(np.random.default_rng(1).standard_normal(tuple(img.shape)), device=img.device)
        full = plan.adjoint(w)
        plan.want = 0b11
        part = plan.adjoint(w)
        for k in ('leaf_flux', 'leaf_jac', 'leaf_size', 'leaf_n'):
            a, b = part[k].cpu().numpy(), full[k].cpu().numpy()
            scale = np.abs(b[:, :2]).max()
            assert np.abs(a[:, :2] - b[:, :2]).max() <= tol * scale, (prec, k)
            assert np.all(a[:, 2:] == 0.)
        for k in ('phase_cen', 'phase_fs', 'phase_jac', 'scales'):
            assert np.all(part[k].cpu().numpy() == 0.)


def test_gradients_vs_differenced_reference_drawimage():
    """Adjoint gradients of sum(w * image) for the fit-step model against central differences
    of the reference's own drawImage (tests/golden/reference_grad.npz, step 1e-4): FP64 and
    FP32 adjoints to 1e-4 (natural units, as above)."""
    import os
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'reference_grad.npz'))
    params, w, fd = d['params'], d['w'], d['fd_grad']
    psf = galsim.Convolve(galsim.Moffat(beta=2.5, fwhm=0.8), galsim.Pixel(0.2))
    dev = galsim._lib.Device.torch_device()
    wt = torch.as_tensor(w, device=dev)
    for prec, dt in (('fp64', np.float64), ('fp32', np.float32)):
        m = autodiff.GalaxyModel(psf, 48, 48, 0.2, dtype=dt, precision=prec)
        p = torch.as_tensor(params, device=dev, dtype=torch.float64).requires_grad_(True)
        (m(p).double() * wt).sum().backward()
        _assert_grad_close(p.grad.cpu().numpy(), fd, params, 1e-4)
