#!/usr/bin/env python
"""Benchmark of the batched FFT drawing path (stamps/s) on B200.

Workload (the batched-forward configuration): 4096 stamps, seed 1234.  Each stamp is
Sersic(n ~ U[0.5, 4], hlr lognormal(median 0.5", sigma_ln 0.3), flux lognormal(median 1e4,
sigma_ln 1)) sheared by g1, g2 ~ N(0, 0.2) clipped to |g| < 0.7, convolved with
Kolmogorov(fwhm ~ U[0.6, 0.9]") and Pixel(0.2), drawn with drawImage(method='fft') at scale
0.2 into an automatically sized float32 image, default GSParams (FFT sizes 128/192/256).
Synthetic parameters; there is no dataset.

One step = the whole device path for the batch: FP64 Sersic FT tables and leaf sizing on the
GPU, GalSim's integer sizing on the host, and the fused k-space/wrap/FFT/crop kernels.
`value` is stamps/s with the flattened inputs resident in HBM; `e2e` is the same through
the public API (galsim_b200.draw_batch) from host parameter arrays to host pixels.

`grad_evals` is the differentiable fit step: 1024 stamps of 48x48 of
Convolve(Sersic(n, hlr, flux).shear(g1, g2).shift(dx, dy), Moffat(2.5, fwhm=0.8), Pixel(0.2)),
chi^2 against a noisy target (SNR 50) and its gradient in the seven parameters through the
adjoint kernels (galsim_b200.autodiff), timed from host parameters to host gradients.
Both carry the plain one-stamp-per-call rate of the same path beside them.

`noise` applies the reference's CCDNoise to every stamp on the device (one seeded stream per
stamp), beside the reference's C++ deviates on the host cores.

`interp_psf` is the InterpolatedImage workload: the same 4096 galaxies convolved with one
image PSF (a 32 x 32 effective-PSF image, quintic interpolants) drawn with
method='no_pixel': device step, draw stage, k-image build, e2e and the reference's C++ on
the host cores for the same stamps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_DEFAULT = 4096
SCALE = 0.2


def workload_params(B=B_DEFAULT, seed=1234):
    """Per-stamp parameters, sampled stamp by stamp in the order n, hlr, flux, g1, g2, psf."""
    rng = np.random.default_rng(seed)
    p = np.zeros((B, 6))
    for i in range(B):
        n = rng.uniform(0.5, 4.0)
        hlr = math.exp(math.log(0.5) + 0.3 * rng.normal())
        flux = math.exp(math.log(1e4) + 1.0 * rng.normal())
        g1 = rng.normal(0., 0.2)
        g2 = rng.normal(0., 0.2)
        g = math.hypot(g1, g2)
        if g >= 0.7:
            g1 *= 0.699 / g
            g2 *= 0.699 / g
        fwhm = rng.uniform(0.6, 0.9)
        p[i] = (n, hlr, flux, g1, g2, fwhm)
    return p


FIT_B = 1024
FIT_NX = 48


def fit_params(B=FIT_B, seed=4321):
    """Fit-step parameters (flux, hlr, n, g1, g2, dx, dy): n ~ U[1, 3], hlr ~ U[0.3, 1.2]",
    flux lognormal(median 1e4, sigma_ln 0.5), g1, g2 ~ N(0, 0.1), dx, dy ~ N(0, 0.1)"; the target
    is drawn at parameters perturbed by 3% (0.02 absolute for g and the centroid) plus Gaussian
    noise at SNR 50."""
    rng = np.random.default_rng(seed)
    true = np.stack([1e4 * np.exp(rng.normal(0., 0.5, B)), rng.uniform(0.3, 1.2, B),
                     rng.uniform(1., 3., B), rng.normal(0., 0.1, B), rng.normal(0., 0.1, B),
                     rng.normal(0., 0.1, B), rng.normal(0., 0.1, B)], -1)
    pert = true * (1. + rng.normal(0., 0.03, true.shape)) + \
        rng.normal(0., 0.02, true.shape) * np.array([0., 0., 0., 1., 1., 1., 1.])
    return true, pert, rng


def run_fit_step(args, galsim, dev, steps, warmup):
    """grad-evals/s of the chi^2 fit step: 1024 stamps of 48x48, Convolve(Sersic(n, hlr, flux)
    .shear(g1, g2).shift(dx, dy), Moffat(2.5, fwhm=0.8), Pixel(0.2)); one grad-eval = forward
    draw + chi^2 + adjoint for one stamp (FP32 kernels, FP64 tables and sizing on the GPU)."""
    import torch
    from galsim_b200 import autodiff
    psf = galsim.Convolve(galsim.Moffat(beta=2.5, fwhm=0.8), galsim.Pixel(SCALE))
    true, pert, rng = fit_params()
    B = len(pert)
    m64 = autodiff.GalaxyModel(psf, FIT_NX, FIT_NX, SCALE, dtype=np.float64, precision='fp64')
    timg = m64(torch.as_tensor(true, device=dev)).detach()
    sigma = torch.sqrt((timg ** 2).sum(dim=(1, 2))) / 50.
    target = (timg + sigma[:, None, None] * torch.as_tensor(
        rng.standard_normal(tuple(timg.shape)), device=dev)).float()
    model = autodiff.GalaxyModel(psf, FIT_NX, FIT_NX, SCALE, dtype=np.float32, precision='fp32')
    isig = (1. / sigma).float()[:, None, None]

    def step(p_host):
        p = torch.as_tensor(p_host, device=dev).requires_grad_(True)
        chi2 = (((model(p) - target) * isig) ** 2).sum()
        chi2.backward()
        return p.grad

    for _ in range(warmup):
        step(pert)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        g = step(pert).cpu()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    # plain: one stamp per call
    n_plain = 16
    for i in range(2):
        step(pert[i:i + 1])
    torch.cuda.synchronize(dev)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    for i in range(n_plain):
        p = torch.as_tensor(pert[i:i + 1], device=dev).requires_grad_(True)
        (((model(p) - target[i:i + 1]) * isig[i:i + 1]) ** 2).sum().backward()
    p1.record()
    torch.cuda.synchronize(dev)
    plain = n_plain / (p0.elapsed_time(p1) * 1e-3)
    N = model.plan.last.N
    return {'value': B / (ms * 1e-3), 'unit': 'grad-evals/s', 'ms_per_step': ms, 'stamps': B,
            'workload': 'sersic_moffat25_pixel_48x48_1024_seed4321 chi2 gradient (flux, hlr, n, g1, g2, dx, dy)',
            'fft_sizes': sorted(set(int(v) for v in N)),
            'timed': 'host parameters -> forward + chi2 + adjoint -> host gradients',
            'plain_one_stamp_per_launch': {'value': plain, 'unit': 'grad-evals/s', 'sample': n_plain}}


MIX_B = 16384
LARGE_B = 64


def mixed_params(B=MIX_B, seed=2468):
    """Bulge + disk batch: total flux lognormal(median 1e4, sigma_ln 0.5), bulge fraction
    U[0, 0.6], bulge hlr lognormal(median 0.4", sigma_ln 0.3), disk hlr lognormal(median 0.8",
    sigma_ln 0.3), independent shears N(0, 0.2) clipped to |g| < 0.6, Moffat beta ~ U[2.5, 4.5]
    and fwhm ~ U[0.5, 1.0]"."""
    rng = np.random.default_rng(seed)
    flux = 1e4 * np.exp(rng.normal(0., 0.5, B))
    bf = rng.uniform(0., 0.6, B)
    bh = 0.4 * np.exp(rng.normal(0., 0.3, B))
    dh = 0.8 * np.exp(rng.normal(0., 0.3, B))

    def shear():
        g = rng.normal(0., 0.2, (B, 2))
        a = np.hypot(g[:, 0], g[:, 1])
        return g * np.where(a >= 0.6, 0.599 / np.maximum(a, 1e-300), 1.)[:, None]

    g_b, g_d = shear(), shear()
    beta = rng.uniform(2.5, 4.5, B)
    fwhm = rng.uniform(0.5, 1.0, B)
    return dict(flux=flux, bf=bf, bh=bh, dh=dh, g_b=g_b, g_d=g_d, beta=beta, fwhm=fwhm)


def mixed_object(galsim, m, gsp):
    bulge = galsim.Sersic(n=4., half_light_radius=m['bh'], flux=m['flux'] * m['bf'], gsparams=gsp) \
        .shear(g1=m['g_b'][:, 0], g2=m['g_b'][:, 1])
    disk = galsim.Exponential(half_light_radius=m['dh'], flux=m['flux'] * (1. - m['bf']), gsparams=gsp) \
        .shear(g1=m['g_d'][:, 0], g2=m['g_d'][:, 1])
    psf = galsim.Moffat(beta=m['beta'], fwhm=m['fwhm'], gsparams=gsp)
    return galsim.Convolve(galsim.Add(bulge, disk), psf, galsim.Pixel(SCALE, gsparams=gsp))


def run_mixed(galsim, dev, steps, warmup):
    """Mixed-size batch: stamps/s forward and forward+adjoint (gradients of the bulge and disk
    records -- flux, Jacobian, size, Sersic n -- for a random cotangent), automatically sized
    stamps with minimum_fft_size=32 (FFT sizes 32..1024)."""
    import torch
    from galsim_b200 import _lib
    gsp = galsim.GSParams(minimum_fft_size=32)
    m = mixed_params()
    plan = galsim.plan_batch(mixed_object(galsim, m, gsp), scale=SCALE, dtype=np.float32)
    prog = plan.prog
    prog.need_dn = True
    st = galsim.run_batch(plan)
    cot = torch.randn(st.flat.numel(), device=dev, dtype=torch.float32)

    def fwd():
        return galsim.run_batch(plan)

    def fwd_adj():
        s = galsim.run_batch(plan)
        return prog.adjoint_stamps(cot[:s.flat.numel()], _lib.F32, want=0b11)   # bulge, disk

    out = {}
    for name, fn in (('forward', fwd), ('forward_adjoint', fwd_adj)):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        out[name] = MIX_B / (e0.elapsed_time(e1) / steps * 1e-3)
    u, c = np.unique(st.N, return_counts=True)
    return {'value': out['forward'], 'unit': 'stamps/s', 'forward_adjoint': out['forward_adjoint'],
            'forward_adjoint_unit': 'grad-evals/s', 'stamps': MIX_B,
            'workload': 'bulge_disk_moffat_gen_pixel_16384_seed2468 (Sersic n=4 + Exponential, Moffat beta U[2.5,4.5])',
            'gsparams': 'minimum_fft_size=32', 'fft_sizes': dict(zip(map(int, u), map(int, c)))}


# Chromatic stage: a bulge + disk batch with one SED per component (tabulated, photons/nm),
# convolved with an atmospheric PSF whose size and centroid depend on wavelength, drawn through a
# tabulated bandpass.  Synthetic spectra and throughput stand in for the reference's share/ files.
CHROM_B = 4096
CHROM_SED_BULGE = ([300., 400., 500., 600., 700., 800., 900., 1100.], [0.3, 0.6, 1.0, 1.4, 1.6, 1.7, 1.7, 1.6])
CHROM_SED_DISK = ([300., 400., 500., 600., 700., 800., 900., 1100.], [2.0, 1.8, 1.4, 1.1, 0.9, 0.8, 0.7, 0.6])
CHROM_BP = ([400., 420., 440., 460., 480., 500., 520., 540., 560., 580., 600.],
            [0.0, 0.35, 0.62, 0.71, 0.74, 0.76, 0.75, 0.70, 0.52, 0.2, 0.0])


def chromatic_object(galsim, m):
    sb = galsim.SED(galsim.LookupTable(*CHROM_SED_BULGE, interpolant='linear'), 'nm', 'fphotons')
    sd = galsim.SED(galsim.LookupTable(*CHROM_SED_DISK, interpolant='linear'), 'nm', 'fphotons')
    bulge = galsim.Sersic(n=4., half_light_radius=m['bh'], flux=m['flux'] * m['bf'] * 1e-2) \
        .shear(g1=m['g_b'][:, 0], g2=m['g_b'][:, 1]) * sb
    disk = galsim.Exponential(half_light_radius=m['dh'], flux=m['flux'] * (1. - m['bf']) * 1e-2) \
        .shear(g1=m['g_d'][:, 0], g2=m['g_d'][:, 1]) * sd
    psf = galsim.ChromaticAtmosphere(galsim.Kolmogorov(fwhm=0.7), 500., zenith_angle=30. * galsim.degrees,
                                     parallactic_angle=20. * galsim.degrees)
    bp = galsim.Bandpass(galsim.LookupTable(*CHROM_BP, interpolant='linear'), 'nm')
    return galsim.Convolve(galsim.Add(bulge, disk), psf), bp


def run_chromatic(galsim, dev, steps, warmup):
    """Chromatic batch: 4096 bulge + disk galaxies (two SEDs) through ChromaticAtmosphere and a
    bandpass, 32 x 32 stamps.  One step = both terms' effective PSFs (their wavelengths drawn in
    real space as one batch each, integrated on the device, turned into InterpolatedImages) and
    the two batched galaxy draws, summed on the device."""
    import torch
    m = mixed_params(CHROM_B, seed=1357)
    obj, bp = chromatic_object(galsim, m)

    def step():
        return galsim.draw_batch(obj, nx=32, ny=32, scale=SCALE, bandpass=bp)

    for _ in range(warmup):
        st = step()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        st = step()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    from galsim_b200.sed import combine_wave_list
    return {'value': CHROM_B / (ms * 1e-3), 'unit': 'stamps/s', 'ms_per_step': ms, 'stamps': CHROM_B,
            'wavelengths_per_integral': int(len(combine_wave_list(obj.obj_list[1] * obj.obj_list[0].obj_list[0].sed,
                                                                  bp)[0])),
            'workload': 'bulge_disk_2sed_chromatic_atmosphere_kolmogorov_32x32_4096_seed1357',
            'timed': 'galsim_b200.draw_batch(chromatic object, bandpass): effective PSFs + batched draws '
                     '(host orchestration included)',
            'flux_check': float(np.median(st.added_flux))}


def _ref_noise_worker(args):
    stamps, seeds = args
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import ctypes
    import ref_draw as R
    L = R.lib()
    L.gsref_ccd_noise.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_longlong, ctypes.c_long,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double]
    t = time.perf_counter()
    for a, sd in zip(stamps, seeds):
        a = np.ascontiguousarray(a, dtype=np.float64)
        L.gsref_ccd_noise(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size, int(sd),
                          NOISE_SKY, NOISE_GAIN, NOISE_READ)
    return time.perf_counter() - t


NOISE_SKY, NOISE_GAIN, NOISE_READ = 100., 1.5, 5.


def run_fits(galsim, st, reps=3):
    """FITS stage: the multi-extension file image of the main workload's 4096 stamps (one HDU
    per stamp), assembled on the device by gsb_fits_pack and read back once, against the host
    writer given the same stamps as host Images (formatting every header and byte-swapping every
    pixel on the host).  Both end as the bytes of the file; the disk write is not timed."""
    from galsim_b200 import fits
    st._fits_image()                                   # warm (the page-locked buffer)
    t0 = time.perf_counter()
    for _ in range(reps):
        dev_image = st._fits_image()                   # what StampBatch.writeMulti writes
    dev_ms = (time.perf_counter() - t0) / reps * 1e3
    dev_bytes = dev_image.tobytes()
    t0 = time.perf_counter()
    ims = st.images()
    hl = fits.HDUList()
    for im in ims:
        hl.append(fits._image_hdu(im, len(hl) == 0))
    host_bytes = fits._file_bytes(hl)
    host_ms = (time.perf_counter() - t0) * 1e3
    return {'file_bytes': len(dev_bytes), 'device_ms': dev_ms, 'host_ms': host_ms,
            'device_gb_per_s': len(dev_bytes) / (dev_ms * 1e-3) / 1e9,
            'identical': dev_bytes == host_bytes,
            'workload': 'writeMulti file image of the %d stamps (FP32), device pack + one read-back '
                        'vs host formatting and byte swap from host Images' % len(st)}


def run_noise(galsim, dev, st, steps, warmup, cpu=True):
    """Noise stage: CCDNoise(sky 100, gain 1.5 e-/ADU, read noise 5 e-) on every stamp of the
    main workload's batch, stamp i with its own BaseDeviate(1 + i) (the reference's Poisson and
    Gaussian streams), on the device before any copy to the host."""
    import torch
    from galsim_b200.batch import StampBatch
    noise = galsim.CCDNoise(sky_level=NOISE_SKY, gain=NOISE_GAIN, read_noise=NOISE_READ)
    B = len(st)
    seeds = 1 + np.arange(B)
    work = st.flat.clone()
    sb = StampBatch(work, st.offsets, st.nx, st.ny, None, None, None, None, None, st.dtype, st.scale, None)
    for _ in range(warmup):
        work.copy_(st.flat)
        sb.addNoise(noise, seeds)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot = 0.
    for _ in range(steps):
        work.copy_(st.flat)
        e0.record()
        sb.addNoise(noise, seeds)
        e1.record()
        torch.cuda.synchronize(dev)
        tot += e0.elapsed_time(e1)
    ms = tot / steps
    npix = int((np.asarray(st.nx) * np.asarray(st.ny)).sum())
    out = {'value': B / (ms * 1e-3), 'unit': 'stamps/s', 'ms': ms, 'pixels': npix,
           'mpix_per_s': npix / (ms * 1e-3) / 1e6,
           'workload': 'CCDNoise(sky 100, gain 1.5, read noise 5) on the 4096 stamps of the main '
                       'workload, BaseDeviate(1 + i) per stamp, one warp per stamp',
           'timed': 'gsb_add_noise including the per-call host setup (stamp records, scratch)'}
    if cpu:
        import multiprocessing as mp
        sys.path.insert(0, os.path.join(ROOT, 'oracle'))
        import ref_draw as R
        if R.available():
            cores = os.cpu_count() or 1
            n = min(B, 64 * cores)
            arrs = [st.array(i).astype(np.float64) for i in range(n)]
            chunks = [(arrs[i::cores], seeds[:n][i::cores]) for i in range(cores)]
            ctx = mp.get_context('spawn')
            with ctx.Pool(cores) as pool:
                pool.map(_ref_noise_worker, chunks[:1])        # warm the imports
                t = time.perf_counter()
                pool.map(_ref_noise_worker, chunks)
                wall = time.perf_counter() - t
            out['cpu_baseline'] = {'value': n / wall, 'unit': 'stamps/s', 'cores': cores, 'kind': 'reference',
                                   'sample': '%d leading stamps (reference C++ PoissonDeviate / '
                                             'GaussianDeviate, one process per core)' % n}
    return out


INTERP_PSF_SIZE = 32


def interp_psf_image(galsim):
    """The PSF image of the image-PSF workload: Kolmogorov(fwhm=0.7") x Pixel(0.2") drawn by this
    library into 32 x 32 float64 pixels (an effective PSF image, as a PSF model would give)."""
    return galsim.Kolmogorov(fwhm=0.7).drawImage(nx=INTERP_PSF_SIZE, ny=INTERP_PSF_SIZE, scale=SCALE,
                                                 dtype=np.float64).array.copy()


def interp_object(galsim, params, psf):
    n, hlr, flux, g1, g2 = [np.ascontiguousarray(params[:, i]) for i in range(5)]
    gal = galsim.Sersic(n=n, half_light_radius=hlr, flux=flux).shear(g1=g1, g2=g2)
    return galsim.Convolve(gal, psf)


def run_interp(galsim, dev, params, steps, warmup, cpu=True):
    """Image-PSF workload: the 4096 galaxies of the main workload (Sersic, sheared) convolved
    with one InterpolatedImage PSF (the 32 x 32 effective-PSF image, quintic interpolants,
    pad_factor 4 -> a 128 x 128 k-image), drawn with method='no_pixel' at automatic sizes.
    Reports the device-timed step, the draw graph alone, the k-image build (1 and 256
    images), e2e through draw_batch, and the reference C++ on the host cores."""
    import torch
    arr = interp_psf_image(galsim)
    psf = galsim.InterpolatedImage(galsim.Image(arr, scale=SCALE))
    plan = galsim.plan_batch(interp_object(galsim, params, psf), scale=SCALE, dtype=np.float32,
                             method='no_pixel')
    for _ in range(warmup):
        st = galsim.run_batch(plan)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        st = galsim.run_batch(plan)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    B = plan.prog.B
    gs = getattr(plan.prog, '_graph_state', None)
    k_ms = None
    if gs is not None and gs.get('graph') is not None:
        reps = max(steps, 10)
        e0.record()
        for _ in range(reps):
            gs['graph'].replay()
        e1.record()
        torch.cuda.synchronize(dev)
        k_ms = e0.elapsed_time(e1) / reps
    # e2e: host parameters -> objects -> draw_batches -> host pixels and fluxes (one PSF object,
    # reused; the next step planned on a worker thread, each step read on a copy stream), after
    # warm-up steps that make the one-time allocations
    for _ in galsim.draw_batches((interp_object(galsim, params, psf) for _ in range(max(warmup, 2))),
                                 scale=SCALE, dtype=np.float32, method='no_pixel'):
        pass
    es, ee = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    es.record()
    for sb, pix, flux in galsim.draw_batches((interp_object(galsim, params, psf) for _ in range(steps)),
                                             scale=SCALE, dtype=np.float32, method='no_pixel'):
        pass
    ee.record()
    torch.cuda.synchronize(dev)
    e2e_ms = es.elapsed_time(ee) / steps
    # k-image build: one 32 x 32 source, and 256 distinct ones
    from galsim_b200.program import Program
    build = {}
    for nimg in (1, 256):
        imgs = [galsim.Image(arr * (1. + 1e-3 * i), scale=SCALE) for i in range(nimg)]
        iib = galsim.InterpolatedImage(imgs if nimg > 1 else imgs[0])
        pr = Program(galsim.Convolve(galsim.Gaussian(sigma=np.full(nimg, 0.5)), iib))
        pr.upload()
        pr._build_images()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(5):
            pr.tables._image_key = None
            pr._build_images()
        torch.cuda.synchronize(dev)
        build['%d_images_ms' % nimg] = (time.perf_counter() - t0) / 5 * 1e3
    u, c = np.unique(st.N, return_counts=True)
    out = {'value': B / (ms * 1e-3), 'unit': 'stamps/s', 'stamps': B, 'ms_per_step': ms,
           'draw_graph_ms': k_ms,
           'e2e': {'value': B / (e2e_ms * 1e-3), 'unit': 'stamps/s', 'mode': 'draw_batches, pipelined'},
           'k_image_build': build,
           'workload': 'sersic_4096_seed1234 x InterpolatedImage(32x32 Kolmogorov(0.7) x Pixel(0.2) '
                       'image, quintic), method=no_pixel',
           'fft_sizes': dict(zip(map(int, u), map(int, c)))}
    if cpu:
        ref = cpu_interp_rate(params, arr)
        if ref is not None:
            out['cpu_baseline'] = ref
    return out


def run_large(galsim, dev):
    """Large-stamp precision study: 64 stamps of Sersic(n ~ U[4, 6], hlr ~ U[2, 5]") x
    Airy(lam/D = 0.1", obscuration 0.3) x Pixel(0.05), default GSParams (folding 5e-3, maxk
    1e-3), automatic sizes; FP32 and FP64 renders, FP32 error per stamp against FP64 (which
    matches the reference to 1e-9 x peak on the large-FFT fixtures)."""
    import torch
    rng = np.random.default_rng(97531)
    n = rng.uniform(4., 6., LARGE_B)
    hlr = rng.uniform(2., 5., LARGE_B)
    flux = np.full(LARGE_B, 1e5)
    times = {'fp32': 0., 'fp64': 0.}
    N_all, err, ferr, npix = [], [], [], []
    chunk = 8
    for c0 in range(0, LARGE_B, chunk):
        sub = galsim.Convolve(galsim.Sersic(n=n[c0:c0 + chunk], half_light_radius=hlr[c0:c0 + chunk],
                                            flux=flux[c0:c0 + chunk]),
                              galsim.Airy(lam_over_diam=0.1, obscuration=0.3), galsim.Pixel(0.05))
        res = {}
        for prec, dt in (('fp32', np.float32), ('fp64', np.float64)):
            plan = galsim.plan_batch(sub, scale=0.05, dtype=dt, precision=prec)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            sb = galsim.run_batch(plan)
            e1.record()
            torch.cuda.synchronize(dev)
            times[prec] += e0.elapsed_time(e1) * 1e-3
            res[prec] = sb
        a, b = res['fp32'], res['fp64']
        fa, fb = a.added_flux, b.added_flux
        for i in range(len(a)):
            o, m_ = int(a.offsets[i]), int(a.nx[i] * a.ny[i])
            d = (a.flat[o:o + m_].double() - b.flat[o:o + m_]).abs().max().item()
            pk = b.flat[o:o + m_].abs().max().item()
            err.append(d / pk)
            ferr.append(abs(fa[i] - fb[i]) / abs(fb[i]))
            N_all.append(int(a.N[i]))
            npix.append(m_)
        del res, a, b
    return {'value': LARGE_B / times['fp32'], 'unit': 'stamps/s', 'fp64_stamps_per_s': LARGE_B / times['fp64'],
            'stamps': LARGE_B, 'workload': 'sersic_n4to6_airy_pixel005_64_seed97531',
            'fft_sizes': N_all, 'pixels': npix,
            'fp32_max_abs_err_over_peak': err, 'fp32_flux_rel_err': ferr,
            'reference_check': 'FP64 renders match the reference C++ to 1e-9 x peak on tests/golden/reference_large.npz'}


def fp32_error_vs_reference(st):
    """Max |diff| / peak and flux error of the leading stamps of a drawn batch against the
    reference's drawImage of the same stamps (tests/golden/reference_configs.npz: its centred
    blocks and strided grids, made by tests/golden/make_golden.py --configs-only)."""
    path = os.path.join(ROOT, 'tests', 'golden', 'reference_configs.npz')
    if not os.path.exists(path):
        return None
    ref = np.load(path)
    shapes = ref['c2_shape']
    block, stride = int(ref['cfg_block']), int(ref['cfg_stride'])
    bo = go = 0
    errs, ferrs = [], []
    for i in range(min(len(shapes), len(st))):
        a = st.array(i)
        if a.shape != tuple(shapes[i]):
            return {'error': 'stamp %d shape %s differs from the reference %s' % (i, a.shape, tuple(shapes[i]))}
        b = min(block, *a.shape)
        y0, x0 = (a.shape[0] - b) // 2, (a.shape[1] - b) // 2
        blk, grd = a[y0:y0 + b, x0:x0 + b].ravel(), a[::stride, ::stride].ravel()
        rb, rg = ref['c2_block'][bo:bo + blk.size], ref['c2_grid'][go:go + grd.size]
        bo += blk.size
        go += grd.size
        pk = float(ref['c2_peak'][i])
        errs.append(max(np.abs(blk.astype(float) - rb).max(), np.abs(grd.astype(float) - rg).max()) / pk)
        fr = float(ref['c2_flux'][i])
        ferrs.append(abs(float(st.added_flux[i]) - fr) / abs(fr))
    return {'stamps': len(errs), 'max_abs_over_peak_median': float(np.median(errs)),
            'max_abs_over_peak_max': float(np.max(errs)), 'flux_rel_median': float(np.median(ferrs)),
            'flux_rel_max': float(np.max(ferrs)),
            'against': "the reference's drawImage of the same stamps (centred 24x24 block and every "
                       "7th pixel of each stamp, tests/golden/reference_configs.npz)"}


def write_detail(detail):
    """Per-stamp lists beside the JSON line (gpurun_out/bench_detail.json when that folder
    exists, else bench_detail.json in the working directory)."""
    d = os.path.join(os.getcwd(), 'gpurun_out')
    path = os.path.join(d if os.path.isdir(d) else os.getcwd(), 'bench_detail.json')
    try:
        with open(path, 'w') as f:
            json.dump(detail, f)
    except OSError:
        pass


def gpu_object(galsim, p):
    gal = galsim.Sersic(n=p[:, 0], half_light_radius=p[:, 1], flux=p[:, 2]).shear(g1=p[:, 3], g2=p[:, 4])
    return galsim.Convolve(gal, galsim.Kolmogorov(fwhm=p[:, 5]), galsim.Pixel(SCALE))


# DRAM bytes of one step's draw kernels (ncu, one-pass metrics, this workload at its own
# automatic sizes; profiles/draw_fused_kernel_dram_bench_step_4096.md): reads, writes, and the
# global stores the SMs issue (stamps plus the N >= 256 buckets' W slabs, which stay in L2).
DRAW_STEP_DRAM_READ = 37439488
DRAW_STEP_DRAM_WRITE = 63917824
DRAW_STEP_STORES = 285221408
# FP64 pipe and issue utilisation of the Sersic table kernel (ncu --set full, round 5 of a
# 4096-table build; profiles/sersic_nodes_pair_kernel_4096_tables.md)
TABLES_FP64_PIPE = 0.446
TABLES_ISSUE_ACTIVE = 0.747


def table_build_launches(n_values, gsp_kvalue_accuracy=1e-5, table_spacing=1.):
    """Kernel launches of one Sersic table build (gsb_sersic_tables_build): setup, scan init,
    one (nodes, scan) pair per round of 64 ln k nodes over the table stride (kTableRound in
    csrc/gsb_tables.cu), and the finalize.
    The stride is the node count of the largest n (sersic_stride in csrc/gsb_tables.cu)."""
    nmax = float(np.max(n_values))
    kderiv6 = math.exp(math.lgamma(8. * nmax) - math.lgamma(2. * nmax)) / 2304.
    kmin = (gsp_kvalue_accuracy / kderiv6) ** (1. / 6.)
    dlogk = table_spacing * math.sqrt(math.sqrt(gsp_kvalue_accuracy / 10.))
    stride = int((math.log(500.) - (math.log(kmin) - 0.001)) / dlogk) + 4
    return 3 + 2 * ((stride + 63) // 64)


def algorithmic_bytes(N, nx, ny):
    """Per-stamp algorithmic bytes of the FFT drawing path at FP32 storage: k-grid write,
    FFT read, FFT write, fold read, stamp write (8 H + 8 H + 4 N^2 + 4 nx ny + 4 nx ny,
    H = N (N/2 + 1))."""
    N = np.asarray(N, np.float64)
    H = N * (N // 2 + 1)
    return 16. * H + 4. * N * N + 8. * np.asarray(nx, np.float64) * np.asarray(ny, np.float64)


class ClockSampler(object):
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        import threading
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.QUERY,
                                          '--format=csv,noheader,nounits', '-lms', '100'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self

        def reader():
            for line in self.proc.stdout:
                if line.strip():
                    self.lines.append(line)
        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        return self

    def wait_first(self, timeout=5.):
        """Block until the sampler has produced its first line (so the timed region is covered)."""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.02)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            self.thread.join(timeout=5)

    def summary(self):
        sm, smax, reasons = [], 0., set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for l in getattr(self, 'lines', []):
            f = [x.strip() for x in l.split(',')]
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': smax or None,
                'reasons': sorted(reasons), 'samples': len(sm),
                'window': 'every 100 ms across the warm-up, the timed steps and the e2e steps'}


def measured_peak_hbm():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    return 6650., 'fallback'


# ---------------------------------------------------------------------------------------------
# CPU reference arm: the reference's C++ drawing arithmetic (oracle/_ref/libgsref.so)
# ---------------------------------------------------------------------------------------------
def _ref_worker(rows, repeat=1):
    """Draw rows with the reference C++ (oracle/_ref/libgsref.so) in this process; with
    repeat=2 the rows are drawn twice and only the second pass is timed (the reference's
    SersicInfo LRU cache then holds every table: the warm-table case)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import ref_draw as R
    t = 0.
    for rep in range(repeat):
        t0 = time.perf_counter()
        for p in rows:
            n, hlr, flux, g1, g2, fwhm = p
            R.draw_image(R.c2_profile(n, hlr, flux, g1, g2, fwhm, SCALE), None, None, SCALE)
        t = time.perf_counter() - t0
    return t


def _ref_warm_worker(rows):
    return _ref_worker(rows, repeat=2)


REF_STEP_STAMPS = 512


def cpu_model():
    try:
        with open('/proc/cpuinfo') as f:
            for line in f:
                if line.startswith('model name'):
                    return line.split(':', 1)[1].strip()
    except OSError:
        pass
    return None


class RefPool(object):
    """The reference's C++ drawing path on every host core: one spawn-started process per
    core (the reference's own pattern, galsim/config/util.py MultiProcess), persistent across
    steps.  A step draws REF_STEP_STAMPS consecutive stamps of the batch, split over the
    processes; consecutive steps continue through the batch and wrap around, so eight steps
    cover the 4096 stamps once.  Tables are cold: every stamp has its own Sersic n and a
    process meets each n again only after ~256 other ones (the reference's cache holds 100)."""

    def __init__(self, params):
        import multiprocessing as mp
        sys.path.insert(0, os.path.join(ROOT, 'oracle'))
        import ref_draw as R
        self.available = R.available()
        self.params = params
        self.cores = len(os.sched_getaffinity(0)) if hasattr(os, 'sched_getaffinity') else (os.cpu_count() or 1)
        self.next = 0
        self.pool = mp.get_context('spawn').Pool(self.cores) if self.available else None

    def step(self, S=REF_STEP_STAMPS):
        B = len(self.params)
        idx = (self.next + np.arange(S)) % B
        self.next = int((self.next + S) % B)
        rows = self.params[idx]
        t = time.perf_counter()
        self.pool.map(_ref_worker, [rows[i::self.cores] for i in range(self.cores)])
        return S, time.perf_counter() - t

    def run(self, steps, warmup):
        for _ in range(warmup):
            self.step()
        tot_s, tot_t, per = 0, 0., []
        for _ in range(steps):
            n, t = self.step()
            tot_s += n
            tot_t += t
            per.append(t)
        return tot_s, tot_t, per

    def extras(self):
        """Single-core and warm-table rates and the host CPU, beside the all-core cold rate."""
        one = self.params[:32]
        t1 = self.pool.apply(_ref_worker, (one,))
        rows = self.params[:REF_STEP_STAMPS]
        tw = max(self.pool.map(_ref_warm_worker, [rows[i::self.cores] for i in range(self.cores)]))
        return {'single_core': {'value': len(one) / t1, 'unit': 'stamps/s', 'sample': '32 leading stamps, cold tables, one process'},
                'warm_tables': {'value': len(rows) / tw, 'unit': 'stamps/s', 'cores': self.cores,
                                'sample': '%d leading stamps, each process redrawing its share with '
                                          'the Sersic tables already in the reference\'s cache' % len(rows)},
                'cpu_model': cpu_model(), 'cores_available': os.cpu_count()}

    def close(self):
        if self.pool is not None:
            self.pool.close()
            self.pool.join()


def cpu_reference_rate(params, steps=3, warmup=1, extras=False):
    """stamps/s of the reference's C++ path on all host cores, over `steps` stepped samples of
    REF_STEP_STAMPS stamps of the workload (after `warmup` untimed ones)."""
    rp = RefPool(params)
    if not rp.available:
        return None
    try:
        n, t, per = rp.run(steps, warmup)
        out = {'value': n / t, 'unit': 'stamps/s', 'cores': rp.cores, 'kind': 'reference',
               'sample': '%d steps of %d consecutive stamps of the 4096-stamp batch (cold Sersic tables, '
                         'one process per core, reference C++ with an FP64 Stockham FFT in place of FFTW)'
                         % (steps, REF_STEP_STAMPS),
               'step_ms': [1e3 * v for v in per]}
        if extras:
            out.update(rp.extras())
        return out
    finally:
        rp.close()


def _ref_interp_worker(args):
    rows, psf = args
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import galsim_oracle as O
    import ref_draw as R
    ii = R.RInterpolatedImage(psf, SCALE)
    out = []
    for p in rows:
        n, hlr, flux, g1, g2 = p[:5]
        prof = O.OConvolve(R.RSersic(n, hlr, flux).shear(g1, g2), ii)
        t = time.perf_counter()
        R.draw_image(prof, None, None, SCALE, pixel=False)
        out.append(time.perf_counter() - t)
    return out


def cpu_interp_rate(params, psf, budget_s=8.):
    """stamps/s of the reference's C++ path for the image-PSF workload on all host cores, over
    a bounded leading sample (one InterpolatedImage per process, as a reference user keeps
    one PSF object)."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import ref_draw as R
    if not R.available():
        return None
    cores = os.cpu_count() or 1
    per = _ref_interp_worker((params[:3], psf))
    est = max(np.mean(per[1:]), 1e-3)
    n = int(min(len(params), max(cores, budget_s * cores / est)))
    sample = params[:n]
    chunks = [(sample[i::cores], psf) for i in range(cores)]
    ctx = mp.get_context('spawn')
    with ctx.Pool(cores) as pool:
        t = time.perf_counter()
        pool.map(_ref_interp_worker, chunks)
        wall = time.perf_counter() - t
    return {'value': n / wall, 'unit': 'stamps/s', 'cores': cores, 'kind': 'reference',
            'sample': '%d leading stamps of the 4096-stamp image-PSF batch (reference C++ '
                      'SBInterpolatedImage and SBSersic, one process per core)' % n}


def workload_config(stamps=B_DEFAULT):
    """The workload both arms are quoted on."""
    return {'workload': 'sersic_kolmogorov_pixel_4096_seed1234', 'stamps_per_gpu': stamps,
            'scale': SCALE, 'gsparams': 'default', 'image_dtype': 'float32', 'sizes': 'automatic'}


def run_reference(args):
    """The reference's own CPU implementation of the path (its C++ from oracle/_ref, built
    from the reference sources) on all host cores: W warm-up and K timed steps of
    REF_STEP_STAMPS stamps each, consecutive through the batch."""
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    params = workload_params()
    rp = RefPool(params)
    if not rp.available:
        print(json.dumps({'impl': 'reference', 'unavailable': 'oracle/_ref/libgsref.so is not built'}))
        return
    try:
        n, t, per = rp.run(args.steps, args.warmup)
        ext = rp.extras()
    finally:
        rp.close()
    value = n / t
    cb = {'value': value, 'unit': 'stamps/s', 'cores': rp.cores, 'kind': 'reference',
          'sample': 'each step %d consecutive stamps of the 4096-stamp batch, cycling (cold Sersic '
                    'tables, one process per core, reference C++ with an FP64 Stockham FFT in place '
                    'of FFTW)' % REF_STEP_STAMPS}
    cb.update(ext)
    line = {'metric': 'stamps/s', 'value': value, 'unit': 'stamps/s', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': 1e3 * t / args.steps,
            'stamps_per_step': REF_STEP_STAMPS,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic', 'impl': 'reference', 'config': workload_config(),
            'cpu_baseline': cb,
            'e2e': {'value': value, 'unit': 'stamps/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------
def run_stage(args):
    """Small single-stage runs for profiling (--stage draw | tables | fit | interp | noise |
    fits): no e2e / CPU legs."""
    import torch
    import galsim_b200 as galsim
    from galsim_b200 import _lib
    params = workload_params(args.stamps)
    obj = gpu_object(galsim, params)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.stage == 'chromatic':
        print(json.dumps({'stage': 'chromatic', **run_chromatic(galsim, _lib.Device.torch_device(), args.steps,
                                                                  max(args.warmup, 1))}))
        return
    if args.stage == 'fit':
        from galsim_b200 import autodiff
        psf = galsim.Convolve(galsim.Moffat(beta=2.5, fwhm=0.8), galsim.Pixel(SCALE))
        _, pert, _ = fit_params(min(args.stamps, FIT_B))
        model = autodiff.GalaxyModel(psf, FIT_NX, FIT_NX, SCALE, dtype=np.float32, precision='fp32')
        dev = _lib.Device.torch_device()
        w = torch.randn((len(pert), FIT_NX, FIT_NX), device=dev)

        def step():
            p = torch.as_tensor(pert, device=dev).requires_grad_(True)
            (model(p) * w).sum().backward()

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({'stage': 'fit', 'stamps': len(pert), 'ms_per_step': e0.elapsed_time(e1) / args.steps}))
        return
    if args.stage == 'large':
        dev = _lib.Device.torch_device()
        res = run_large(galsim, dev)
        print(json.dumps({'stage': 'large', 'stamps_per_s': res['value'],
                          'fp64_stamps_per_s': res['fp64_stamps_per_s'],
                          'fp32_flux_rel_err_max': max(res['fp32_flux_rel_err']),
                          'fp32_max_abs_err_over_peak_max': max(res['fp32_max_abs_err_over_peak']),
                          'per_stamp': {k: res[k] for k in ('fft_sizes', 'fp32_flux_rel_err',
                                                             'fp32_max_abs_err_over_peak')}}))
        return
    if args.stage == 'tables':
        t = _lib.Tables()
        n = params[:, 0]
        for _ in range(args.warmup):
            t.build_sersic(n, galsim.GSParams())
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            t.build_sersic(n, galsim.GSParams())
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({'stage': 'tables', 'tables': len(n), 'ms_per_build': e0.elapsed_time(e1) / args.steps}))
        return
    if args.stage == 'fits':
        st = galsim.draw_batch(obj, nx=args.nx, ny=args.nx, scale=SCALE, dtype=np.float32)
        for _ in range(args.warmup):
            st._fits_image()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            img = st._fits_image()
        print(json.dumps({'stage': 'fits', 'stamps': len(st), 'file_bytes': int(img.size),
                          'ms_per_step': (time.perf_counter() - t0) / args.steps * 1e3}))
        return
    if args.stage == 'noise':
        dev = _lib.Device.torch_device()
        st = galsim.draw_batch(obj, nx=args.nx, ny=args.nx, scale=SCALE, dtype=np.float32)
        res = run_noise(galsim, dev, st, args.steps, args.warmup, cpu=False)
        print(json.dumps({'stage': 'noise', 'stamps': len(st), 'ms_per_step': res['ms'],
                          'mpix_per_s': res['mpix_per_s']}))
        return
    if args.stage == 'interp':
        psf = galsim.InterpolatedImage(galsim.Image(interp_psf_image(galsim), scale=SCALE))
        plan = galsim.plan_batch(interp_object(galsim, params, psf), nx=args.nx, ny=args.nx, scale=SCALE,
                                 dtype=np.float32, method='no_pixel')
    else:
        plan = galsim.plan_batch(obj, nx=args.nx, ny=args.nx, scale=SCALE, dtype=np.float32)
    for _ in range(args.warmup):
        st = galsim.run_batch(plan)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        st = galsim.run_batch(plan)
    e1.record()
    torch.cuda.synchronize()
    u, c = np.unique(st.N, return_counts=True)
    print(json.dumps({'stage': args.stage, 'stamps': len(st), 'ms_per_step': e0.elapsed_time(e1) / args.steps,
                      'buckets': dict(zip(map(int, u), map(int, c)))}))


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from galsim_b200 import replicas
    rank, world, local = replicas.rank_info()
    import galsim_b200 as galsim
    from galsim_b200 import _lib
    galsim.set_device(local)
    dev = _lib.Device.torch_device()
    replicas.init('nccl')
    # weak scaling: every rank draws its own batch of the configuration (seed 1234 + rank)
    params = workload_params(args.stamps, seed=1234 + rank)
    obj = gpu_object(galsim, params)
    plan = galsim.plan_batch(obj, scale=SCALE, dtype=np.float32)

    def barrier():
        torch.cuda.synchronize(dev)
        replicas.barrier()

    # Clocks are sampled (every 100 ms) from before the warm-up until after the e2e region; the
    # timed loop starts only once the sampler is producing.
    clk = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        st = galsim.run_batch(plan)
    barrier()
    clk.wait_first()
    # L2 note: the working set (tables ~100 MB, stamp outputs ~50 MB, per-CTA W slabs) is
    # rewritten every step by the table build; inputs are re-read from HBM each step.
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    barrier()
    start.record()
    for _ in range(args.steps):
        st = galsim.run_batch(plan)
    stop.record()
    barrier()
    ms = replicas.max_over_ranks(start.elapsed_time(stop) / args.steps)
    B = plan.prog.B
    value = world * B / (ms * 1e-3)

    # device time of the draw stage alone (every FFT-size bucket of the fused kernel, concurrent
    # on their streams): replays of the step's captured draw graph, back to back
    prog = plan.prog
    N, Nk, nx, ny = st.N, st.Nk, st.nx, st.ny
    nb = len(np.unique(N))
    gstate = getattr(prog, '_graph_state', None)
    ks, ke = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(args.steps, 10)
    torch.cuda.synchronize(dev)
    if gstate is not None and gstate.get('graph') is not None:
        ks.record()
        for _ in range(reps):
            gstate['graph'].replay()
        ke.record()
    else:
        ks.record()
        for _ in range(reps):
            prog.draw_stamps(N, Nk, st.xmin, st.ymin, nx, ny, _lib.F32)
        ke.record()
    torch.cuda.synchronize(dev)
    k_ms = ks.elapsed_time(ke) / reps
    alg = float(algorithmic_bytes(N, nx, ny).sum())
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / (k_ms * 1e-3) / 1e9

    # the Sersic table stage alone (one FP64 table per stamp), CUDA events on its stream
    tables_roof = None
    if prog.tables is not None and prog.sersic_n is not None:
        for _ in range(2):
            prog.tables.build_sersic(prog.sersic_n, prog.gsparams)
        torch.cuda.synchronize(dev)
        ts, te = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ts.record()
        for _ in range(reps):
            prog.tables.build_sersic(prog.sersic_n, prog.gsparams)
        te.record()
        torch.cuda.synchronize(dev)
        t_ms = ts.elapsed_time(te) / reps
        tables_roof = {'bound': 'fp64 issue', 'unit': 'fraction of the FP64 pipe',
                       'kernel': 'sersic_nodes_pair_kernel (+ scan, setup, finalize): %d FP64 Sersic FT tables'
                                 % len(prog.sersic_n),
                       'kernel_ms': t_ms, 'step_share': t_ms / ms,
                       'frac': TABLES_FP64_PIPE, 'issue_active': TABLES_ISSUE_ACTIVE,
                       'frac_source': 'ncu --set full, round 5 of a 4096-table build '
                                      '(profiles/sersic_nodes_pair_kernel_4096_tables.md)'}

    # e2e through the public API: host parameters -> draw_batch -> host pixels.  The warm-up
    # steps make the one-time allocations (the page-locked read-back buffer) before timing.
    def e2e_step():
        o = gpu_object(galsim, params)
        sb = galsim.draw_batch(o, scale=SCALE, dtype=np.float32)
        return sb.host(copy=False), sb.added_flux

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    es, ee = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    es.record()
    for _ in range(args.steps):
        o = gpu_object(galsim, params)
        sb = galsim.draw_batch(o, scale=SCALE, dtype=np.float32)
        pix = sb.host(copy=False)      # read into a reused page-locked host buffer
        flux = sb.added_flux
    ee.record()
    barrier()
    e2e_serial_ms = replicas.max_over_ranks(es.elapsed_time(ee) / args.steps)
    # the same steps pipelined as a catalog run is (galsim_b200.draw_batches): a worker thread
    # builds and uploads step k+1's records while step k's tables and draws run, and step k's
    # pixels are read on a copy stream while step k+1 draws; every step's read-back is inside
    # the timed region (the generator yields each step's host pixels and fluxes)
    for _ in galsim.draw_batches((gpu_object(galsim, params) for _ in range(max(args.warmup, 2))),
                                 scale=SCALE, dtype=np.float32):
        pass
    barrier()
    es.record()
    n_done = 0
    for sb, pix, flux in galsim.draw_batches((gpu_object(galsim, params) for _ in range(args.steps)),
                                             scale=SCALE, dtype=np.float32):
        n_done += 1
    ee.record()
    barrier()
    assert n_done == args.steps
    e2e_ms = replicas.max_over_ranks(es.elapsed_time(ee) / args.steps)
    clk.__exit__(None, None, None)
    L = prog.L
    h2d = B * (L * 136 + len(prog.bld.phases) * 64 + len(prog.bld.scales) * 8 + 32)
    d2h = int(pix.size * 4 + B * 8 + B * L * 16)

    # plain one-stamp-per-launch GPU path on a sample (the metric's denominator)
    n_plain = 64
    sub = gpu_object(galsim, params[:1])
    tp0 = torch.cuda.Event(enable_timing=True)
    tp1 = torch.cuda.Event(enable_timing=True)
    single_objs = [gpu_object(galsim, params[i:i + 1]) for i in range(n_plain)]
    for o in single_objs[:3]:
        galsim.draw_batch(o, scale=SCALE, dtype=np.float32)
    torch.cuda.synchronize(dev)
    tp0.record()
    for o in single_objs:
        galsim.draw_batch(o, scale=SCALE, dtype=np.float32)
    tp1.record()
    torch.cuda.synchronize(dev)
    plain_rate = n_plain / (tp0.elapsed_time(tp1) * 1e-3)

    # FP32 error of the measured path against the reference: the last timed step's first
    # stamps against the same stamps drawn one by one by the reference's own drawImage
    # (tests/golden/reference_configs.npz, the leading 256 stamps of this workload)
    fp32_err = fp32_error_vs_reference(st)

    fit = run_fit_step(args, galsim, dev, max(args.steps, 3), max(args.warmup, 2))
    mixed = run_mixed(galsim, dev, max(args.steps, 3), max(args.warmup, 2)) if not args.no_extra else None
    if not args.no_extra:
        # the large stamps' multi-GB workspaces are allocated inside their timed run_batch
        # calls; releasing the earlier stages' cached blocks first makes those allocations
        # the same as in a process that draws only large stamps
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
    large = run_large(galsim, dev) if not args.no_extra else None
    chrom = run_chromatic(galsim, dev, max(args.steps, 3), max(args.warmup, 2)) if not args.no_extra else None
    interp = (run_interp(galsim, dev, params, max(args.steps, 3), max(args.warmup, 2),
                         cpu=(rank == 0 and world == 1 and not args.no_cpu))
              if not args.no_extra else None)
    # the FITS stage times host-side work too, so it runs before the noise stage's CPU baseline
    # (a pool of one process per core) rather than after it
    fits_stage = run_fits(galsim, st) if not args.no_extra else None
    noise = (run_noise(galsim, dev, st, max(args.steps, 3), max(args.warmup, 2),
                       cpu=(rank == 0 and world == 1 and not args.no_cpu))
             if not args.no_extra else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_rate(params, steps=3, warmup=1, extras=True)

    if rank == 0:
        # per-stamp lists go to a side file; the JSON line keeps their summaries
        detail = {'large_stamps': large, 'step_fft_sizes': [int(v) for v in N]}
        if large is not None:
            large = {k: v for k, v in large.items() if not isinstance(v, list)}
            ls = detail['large_stamps']
            large.update({'fft_sizes': sorted(set(ls['fft_sizes'])),
                          'fp32_max_abs_err_over_peak_max': max(ls['fp32_max_abs_err_over_peak']),
                          'fp32_flux_rel_err_max': max(ls['fp32_flux_rel_err']),
                          'per_stamp': 'bench_detail.json'})
        write_detail(detail)
        line = {
            'metric': 'stamps/s', 'value': value, 'unit': 'stamps/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
            'data': 'synthetic',
            'config': workload_config(B),
            'path': {'fft_sizes': sorted(set(int(v) for v in N)),
                     'parallelism': 'replicas x%d' % world,
                     'draw_stage': ('one CUDA graph replay per step (FFT-size buckets on forked streams)'
                                    if getattr(prog, '_graph_state', None) and prog._graph_state.get('graph')
                                    else 'eager launches'),
                     'autotuned_variants': _lib.tune_report().splitlines(),
                     'l2': 'no flush; per-step table build and stamp outputs exceed L2 reuse'},
            'e2e': {'value': world * B / (e2e_ms * 1e-3), 'unit': 'stamps/s',
                    'h2d_bytes_per_step': int(h2d), 'd2h_bytes_per_step': d2h,
                    'mode': 'host parameters -> draw_batches -> host pixels and fluxes; step k+1 built and '
                            'uploaded on a worker thread while step k runs, step k read back on a copy '
                            'stream while step k+1 draws',
                    'serial_value': world * B / (e2e_serial_ms * 1e-3)},
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'traffic': DRAW_STEP_DRAM_READ + DRAW_STEP_DRAM_WRITE,
                         'traffic_with_stamp_writeback': DRAW_STEP_DRAM_READ + int(pix.size * 4),
                         'traffic_note': 'ncu dram read+write of the step\'s draw kernels at this workload '
                                         '(profiles/draw_fused_kernel_dram_bench_step_4096.md); most stamp '
                                         'writes are still in L2 when each kernel exits, so their write-back '
                                         'is counted in traffic_with_stamp_writeback; the SMs store %d B '
                                         '(stamps + W slabs); algorithmic bytes of the staged path %.0f'
                                         % (DRAW_STEP_STORES, alg),
                         'peak_kind': peak_kind,
                         'kernel': 'draw_fused_kernel, all FFT-size buckets concurrent (one draw-graph replay)',
                         'kernel_ms': k_ms},
            'roofline_tables': tables_roof,
            # per step: the Sersic table build, one leaf-prepare launch, the leaf gather into
            # bucket order, one fused draw per FFT-size bucket and the added-flux scatter
            'gpu_launches': int(args.steps * (table_build_launches(params[:, 0]) + 3 + nb)),
            'fp32_error_vs_reference': fp32_err,
            'mixed_batch': mixed,
            'large_stamps': large,
            'interp_psf': interp,
            'chromatic': chrom,
            'noise': noise,
            'fits': fits_stage,
            'clocks': clk.summary(),
        }
        if cpu is not None:
            line['cpu_baseline'] = cpu
        # the headline's second half last, so that a cut-off tail still shows it
        line['plain_one_stamp_per_launch'] = {'value': plain_rate, 'unit': 'stamps/s', 'sample': n_plain}
        line['grad_evals'] = fit
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='gsb', choices=['gsb', 'reference'])
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline measurement')
    ap.add_argument('--no-extra', action='store_true',
                    help='skip the mixed-batch and large-stamp measurements')
    ap.add_argument('--stamps', type=int, default=B_DEFAULT, help='stamps per GPU (leading subset)')
    ap.add_argument('--nx', type=int, default=None, help='fixed stamp size (default: automatic)')
    ap.add_argument('--stage', default='all', choices=['all', 'draw', 'tables', 'fit', 'interp', 'noise', 'fits', 'large',
                                                       'chromatic'],
                    help="'draw' / 'tables' / 'fit' / 'interp' / 'noise' / 'fits': run only that stage (for profiling)")
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    elif args.stage != 'all':
        run_stage(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
