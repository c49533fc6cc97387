"""GPU parity of InterpolatedImage: the CUDA path (image DFT, stepk / maxk scans, k
interpolation inside the drawing kernels) against fixtures made by the reference
(tests/golden/make_golden.py main_interp) and against the FP64 oracle.

Tolerances as for the analytic profiles: FP32 path max |image difference| <= 1e-5 x peak and
|added_flux difference| <= 1e-6 relative; FP64 path 1e-9 x peak; drawKImage (FP64) 1e-9 of the
largest |value|; stepk and maxk to 1e-14 relative (they come from integer scans).
"""
import numpy as np
import pytest

import galsim_b200 as galsim
import galsim_oracle as O
import make_golden as MG
import specs

pytestmark = pytest.mark.gpu
GOLD = np.load(specs.HERE + '/reference_interp.npz')
specs.load_interp_images(GOLD)


def build(spec):
    return MG.profile(galsim, spec)


@pytest.mark.parametrize('case', MG.INTERP_DRAW_CASES, ids=[c[0] for c in MG.INTERP_DRAW_CASES])
def test_interp_draw_fp32_vs_reference(case):
    name, spec, nx, ny, scale, dt, off = case
    im = build(spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.dtype(dt).type, method='fft',
                               offset=off)
    ref = GOLD['draw_' + name]
    peak = np.abs(ref).max()
    assert im.array.dtype == ref.dtype
    err = np.abs(im.array.astype(float) - ref).max()
    assert err <= 1e-5 * peak, (name, err / peak)
    fref = float(GOLD['draw_' + name + '_flux'])
    assert abs(im.added_flux - fref) <= 1e-6 * abs(fref), (name, im.added_flux, fref)


@pytest.mark.parametrize('case', [c for c in MG.INTERP_DRAW_CASES if c[5] == 'f8'],
                         ids=[c[0] for c in MG.INTERP_DRAW_CASES if c[5] == 'f8'])
def test_interp_draw_fp64_vs_reference(case):
    name, spec, nx, ny, scale, dt, off = case
    im = build(spec).drawImage(nx=nx, ny=ny, scale=scale, dtype=np.float64, method='fft',
                               offset=off, precision='fp64')
    ref = GOLD['draw_' + name]
    assert np.abs(im.array - ref).max() <= 1e-9 * np.abs(ref).max(), name


@pytest.mark.parametrize('case', MG.INTERP_KIMAGE_CASES, ids=[c[0] for c in MG.INTERP_KIMAGE_CASES])
def test_interp_kimage_vs_reference(case):
    name, spec, dk, n = case
    im = build(spec).drawKImage(nx=n, ny=n, scale=dk)
    ref = GOLD['kimg_' + name]
    assert (im.bounds.xmin, im.bounds.ymin) == tuple(GOLD['kimg_' + name + '_xmin'])
    assert np.abs(im.array - ref).max() <= 1e-9 * np.abs(ref).max(), name


def test_interp_sizes_vs_reference():
    for spec, (sk, mk) in zip(MG.INTERP_SIZE_CASES, GOLD['sizes']):
        obj = build(spec)
        assert abs(obj.stepk - sk) <= 1e-14 * sk, (spec, obj.stepk, sk)
        assert abs(obj.maxk - mk) <= 1e-14 * mk, (spec, obj.maxk, mk)


def test_interp_batch_of_images_matches_oracle_per_stamp():
    """A batch of different images (each its own padded frame and k-image) convolved with a
    batch of galaxies, against the oracle stamp by stamp."""
    imgs = [GOLD['img_psf32'], GOLD['img_psf31x33'], GOLD['img_gal24'] * 0.05]
    B = len(imgs)
    hlr = np.array([0.5, 0.7, 0.4])
    g1 = np.array([0.1, -0.2, 0.05])
    ii = galsim.InterpolatedImage([galsim.Image(a, scale=0.2) for a in imgs])
    gal = galsim.Exponential(half_light_radius=hlr, flux=100.).shear(g1=g1, g2=0.05)
    obj = galsim.Convolve(gal, ii)
    stamps = galsim.draw_batch(obj, nx=40, ny=40, scale=0.2)
    for b in range(B):
        oi = O.OInterpolatedImage(imgs[b], 0.2)
        og = O.OConvolve(O.OExponential(hlr[b] / 1.6783469900166605, 100.).shear(g1[b], 0.05), oi)
        ref, flux, N, Nk = O.draw_image(og, 40, 40, 0.2)
        got = np.asarray(stamps.array(b), dtype=float)
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max(), b


def test_interp_shared_image_broadcasts_over_batch():
    """One image (batch 1) convolved with a batch of galaxies: every stamp uses the same
    image slot."""
    psf = galsim.InterpolatedImage(galsim.Image(GOLD['img_psf32'], scale=0.2))
    hlr = np.array([0.4, 0.6, 0.8, 1.0])
    obj = galsim.Convolve(galsim.Sersic(n=2.0, half_light_radius=hlr, flux=50.), psf)
    stamps = galsim.draw_batch(obj, nx=32, ny=32, scale=0.2)
    oi = O.OInterpolatedImage(GOLD['img_psf32'], 0.2)
    for b in range(len(hlr)):
        og = O.OConvolve(O.OSersic(2.0, hlr=hlr[b], flux=50.), oi)
        ref, flux, N, Nk = O.draw_image(og, 32, 32, 0.2)
        got = np.asarray(stamps.array(b), dtype=float)
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max(), b


def test_interp_gradients_with_image_psf_fp64_vs_finite_differences():
    """Fit-step gradients of a galaxy convolved with an InterpolatedImage PSF (the image leaf
    is a constant factor of the adjoint) against FP64 central differences."""
    torch = pytest.importorskip('torch')
    from galsim_b200 import autodiff
    psf = galsim.InterpolatedImage(galsim.Image(GOLD['img_psf32'], scale=0.2))
    model = autodiff.GalaxyModel(psf, 40, 40, 0.2, dtype=np.float64, precision='fp64')
    p0 = np.array([[2e3, 0.6, 1.8, 0.08, -0.05, 0.04, -0.03],
                   [5e3, 0.4, 2.7, -0.1, 0.12, -0.06, 0.02]])
    dev = galsim._lib.Device.torch_device()
    w = torch.as_tensor(np.random.default_rng(5).standard_normal((2, 40, 40)), device=dev)
    p = torch.as_tensor(p0, device=dev, dtype=torch.float64).requires_grad_(True)
    loss = (model(p) * w).sum()
    loss.backward()
    g = p.grad.cpu().numpy()
    for s in range(2):
        for j in range(7):
            h = 1e-6 * (p0[s, j] if j in (0, 1, 2) else 1.)
            vals = []
            for sgn in (1., -1.):
                q = p0.copy()
                q[s, j] += sgn * h
                with torch.no_grad():
                    vals.append(float((model(torch.as_tensor(q, device=dev)) * w).sum()))
            fd = (vals[0] - vals[1]) / (2. * h)
            scale = np.abs(g[s]).max()
            assert abs(g[s, j] - fd) <= 1e-5 * max(abs(fd), 1e-2 * scale), (s, j, g[s, j], fd)
