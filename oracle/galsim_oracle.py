"""ORACLE: FP64 numpy restatement of the reference's FFT drawing path.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline may import this module, and only as the checker; nothing in galsim_b200/ uses it.

It restates, in double precision and with its own tree classes (independent of the
product's host code), the reference algorithm of
    GSObject.drawImage(method='fft' | 'no_pixel')    galsim/gsobject.py:1283-1844
    drawFFT_makeKImage / drawFFT_finish / drawFFT    galsim/gsobject.py:1900-2045
    drawKImage                                       galsim/gsobject.py:2464-2582
    Convolution / Sum / Transformation _drawKImage   convolve.py:420-426, sum.py:341-347,
                                                     transform.py:592-602
    SBProfile::drawK + per-profile fillKImage        src/SBProfile.cpp:383-588 and
                                                     src/SB{Gaussian,Exponential,Sersic,Moffat,
                                                     Kolmogorov,Airy,Box}.cpp
    ApplyKImagePhases                                src/SBTransform.cpp:740-883
    wrapImage (hermx)                                src/Image.cpp:395-727 (pointer walk restated)
    irfft(shift_in, shift_out)                       src/Image.cpp:815-912 (FFTW c2r -> numpy)
    goodFFTSize                                      src/Image.cpp:1141-1153
    SersicInfo (HLR, missing flux, FT table)         src/SBSersic.cpp:301-667
    hankel_inf (Ogata 2005, adaptive h)              src/math/Hankel.cpp:79-249
    natural cubic spline                             src/Table.cpp:553-686
    KolmogorovInfo stepk                             src/SBKolmogorov.cpp:338-420
    Moffat kValue / maxK / stepK                     src/SBMoffat.cpp:163-549
Special functions come from scipy (kv, j0, j1, y0, gammainc, gamma).  Its results are pinned
against fixtures made by the reference itself (tests/golden/).
"""
import math

import numpy as np
from scipy import special

PI = math.pi


# ---------------------------------------------------------------------------------------------
# GSParams
# ---------------------------------------------------------------------------------------------
class OGSParams(object):
    def __init__(self, minimum_fft_size=128, maximum_fft_size=8192, folding_threshold=5.e-3,
                 stepk_minimum_hlr=5, maxk_threshold=1.e-3, kvalue_accuracy=1.e-5,
                 xvalue_accuracy=1.e-5, table_spacing=1, realspace_relerr=1.e-4,
                 realspace_abserr=1.e-6, integration_relerr=1.e-6, integration_abserr=1.e-8,
                 shoot_accuracy=1.e-5):
        self.minimum_fft_size = minimum_fft_size
        self.maximum_fft_size = maximum_fft_size
        self.folding_threshold = folding_threshold
        self.stepk_minimum_hlr = stepk_minimum_hlr
        self.maxk_threshold = maxk_threshold
        self.kvalue_accuracy = kvalue_accuracy
        self.xvalue_accuracy = xvalue_accuracy
        self.table_spacing = table_spacing
        self.integration_relerr = integration_relerr
        self.integration_abserr = integration_abserr
        self.shoot_accuracy = shoot_accuracy


DEFAULT = OGSParams()


# ---------------------------------------------------------------------------------------------
# Root finding: Brent with the reference's bracket expansion (include/galsim/Solve.h)
# ---------------------------------------------------------------------------------------------
def _zbrent(f, a, b, fa, fb, xtol=1e-7, max_steps=40):
    if (fa > 0 and fb > 0) or (fa < 0 and fb < 0):
        raise ValueError("root not bracketed")
    c, fc = b, fb
    d = e = b - a
    for _ in range(max_steps + 1):
        if (fb > 0 and fc > 0) or (fb < 0 and fc < 0):
            c, fc = a, fa
            e = d = b - a
        if abs(fc) < abs(fb):
            a, b, c = b, c, b
            fa, fb, fc = fb, fc, fb
        tol1 = 2. * np.finfo(float).eps * abs(b) + 0.5 * xtol
        xm = 0.5 * (c - b)
        if abs(xm) <= tol1 or fb == 0.:
            return b
        if abs(e) >= tol1 and abs(fa) > abs(fb):
            s = fb / fa
            if a == c:
                p = 2. * xm * s
                q = 1. - s
            else:
                q = fa / fc
                r = fb / fc
                p = s * (2. * xm * q * (q - r) - (b - a) * (r - 1.))
                q = (q - 1.) * (r - 1.) * (s - 1.)
            if p > 0:
                q = -q
            p = abs(p)
            if 2. * p < min(3. * xm * q - abs(tol1 * q), abs(e * q)):
                e = d
                d = p / q
            else:
                d = xm
                e = d
        else:
            d = xm
            e = d
        a, fa = b, fb
        b += d if abs(d) > tol1 else (abs(tol1) if xm >= 0 else -abs(tol1))
        fb = f(b)
    raise RuntimeError("zbrent did not converge")


def solve_upper(f, lo, hi):
    flo, fhi = f(lo), f(hi)
    delta = hi - lo
    for _ in range(1, 40):
        if flo * fhi <= 0:
            break
        lo, flo = hi, fhi
        delta *= 2.
        hi += delta
        fhi = f(hi)
    return _zbrent(f, lo, hi, flo, fhi)


def solve_lower_limit(f, lo, hi, limit):
    fa, fb = f(hi), f(lo)
    a, b = hi, lo
    for _ in range(1, 40):
        if fa * fb <= 0:
            break
        bma, cmb = b - a, limit - b
        a, fa = b, fb
        b = (2. * limit / cmb + a / bma) / (2. / cmb + 1. / bma)
        fb = f(b)
    return _zbrent(f, b, a, fb, fa)


# ---------------------------------------------------------------------------------------------
# Ogata Hankel transform (src/math/Hankel.cpp)
# ---------------------------------------------------------------------------------------------
_ZEROS = {}


def _j0_zeros(n):
    z = _ZEROS.get('z')
    if z is None or len(z) < n:
        s = np.arange(1, max(n, 1024) + 1, dtype=np.float64)
        beta = (s - 0.25) * PI
        ib = 1. / (8. * beta)
        x = beta + ib * (1. + ib * ib * (-124. / 3. + ib * ib * (120928. / 15.)))
        for _ in range(4):
            x = x + special.j0(x) / special.j1(x)
        _ZEROS['z'] = x
        _ZEROS['c'] = special.y0(x) / special.j1(x)
    return _ZEROS['z'][:n], _ZEROS['c'][:n]


_NODES = {}


def _ogata_nodes(h):
    key = h
    if key not in _NODES:
        nmax = int(min(PI / h, 1e6))
        z, c = _j0_zeros(nmax)
        t = h * z / PI
        with np.errstate(over='ignore'):
            psi = t * np.tanh(0.5 * PI * np.sinh(t))
            ch = np.cosh(0.5 * PI * np.sinh(t))
            dpsi = t * 0.5 * PI * np.cosh(t) / (ch * ch) + psi / t
        x = PI / h * psi
        w = c * PI * x * special.j0(x) * dpsi
        _NODES[key] = (x, w)
    return _NODES[key]


def _ogata_sum(f, k, h):
    x, w = _ogata_nodes(h)
    terms = w * f(x / k)
    cs = np.cumsum(terms)
    stop = np.flatnonzero(np.abs(terms) < 1e-15 * np.abs(cs))
    ans = cs[stop[0]] if len(stop) else cs[-1]
    return ans / (k * k)


def hankel_inf(f, k, relerr, abserr):
    """AdaptiveHankelIntegrator::integrate (Hankel.cpp:179-219)."""
    h0 = 1. / 32.
    while h0 > 100. * k:
        h0 *= 0.5
    ans0 = _ogata_sum(f, k, h0)
    h1 = 0.5 * h0
    ans1 = _ogata_sum(f, k, h1)
    err = abs(ans1 - ans0)
    while (err > relerr * ans1 and (err > abserr or abs(ans1) > 2 * abs(ans0))) or ans1 == 0.:
        h0 = h1
        ans0 = ans1
        h1 *= 0.5
        ans1 = _ogata_sum(f, k, h1)
        err = abs(ans1 - ans0)
    return ans1


_GL = {}


def hankel_trunc_exact(f, k, rmax, order=24):
    """int_0^rmax r f(r) J0(k r) dr -- the quantity of math::hankel_trunc
    (src/math/Hankel.cpp:249-255), computed to ~1e-13 relative: Gauss-Legendre (`order` points)
    on the panels between consecutive zeros of J0(k r), the first one graded toward r = 0 in 48
    halvings (where r f(r) may have an integrable cusp, r^(1/n) for a Sersic).  The reference
    integrates the same integral with its own adaptive Gauss-Kronrod-Patterson scheme to relerr
    1e-6, so the two agree to the reference's integration error (this value is the more
    accurate one)."""
    if order not in _GL:
        _GL[order] = np.polynomial.legendre.leggauss(order)
    x, w = _GL[order]
    if k > 0.:
        zs = _j0_zeros(max(16, int(k * rmax / PI) + 8))[0] / k
        zs = zs[zs < rmax]
    else:
        zs = np.zeros(0)
    first = float(zs[0]) if len(zs) else float(rmax)
    grade = first * 2. ** -np.arange(48, 0, -1)
    edges = np.concatenate([grade, [first], zs[1:], [rmax]]) if len(zs) else np.concatenate([grade, [rmax]])
    a, b = edges[:-1], edges[1:]
    h = 0.5 * (b - a)
    r = (a + h)[:, None] + h[:, None] * x[None, :]
    g = r * f(r) * special.j0(k * r)
    return float(np.sum(h[:, None] * w[None, :] * g))


# ---------------------------------------------------------------------------------------------
# Natural cubic spline (src/Table.cpp:553-686)
# ---------------------------------------------------------------------------------------------
class Spline(object):
    def __init__(self, args, vals):
        self.x = np.asarray(args, float)
        self.y = np.asarray(vals, float)
        n = len(self.x)
        y2 = np.zeros(n)
        if n == 3:
            y2[1] = 3. * ((self.y[2] - self.y[1]) / (self.x[2] - self.x[1]) -
                          (self.y[1] - self.y[0]) / (self.x[1] - self.x[0])) / (self.x[2] - self.x[0])
        elif n > 3:
            x, y = self.x, self.y
            c = np.zeros(n)
            for i in range(1, n - 1):
                y2[i] = 6. * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]))
            bb = 2. * (x[2] - x[0])
            for i in range(1, n - 1):
                y2[i] /= bb
                if i == n - 2:
                    break
                a = x[i + 1] - x[i]
                c[i - 1] = a / bb
                bb = 2. * (x[i + 2] - x[i]) - a * c[i - 1]
                y2[i + 1] -= a * y2[i]
            for i in range(n - 3, 0, -1):
                y2[i] -= c[i - 1] * y2[i + 1]
        self.y2 = y2
        self.da = (self.x[-1] - self.x[0]) / (n - 1)
        # ArgVec (Table.cpp:64-130): equal spacing to 1% of a step gives the direct index,
        # otherwise the first argument above a (std::upper_bound)
        self.equal = bool(np.all(np.abs((self.x - self.x[0]) / self.da - np.arange(n)) <= 0.01))

    def __call__(self, a):
        a = np.asarray(a, float)
        n = len(self.x)
        if self.equal:
            i = np.ceil((a - self.x[0]) / self.da).astype(int)
        else:
            i = np.searchsorted(self.x, a, side='right')
        i = np.clip(i, 1, n - 1)
        h = self.x[i] - self.x[i - 1]
        aa = self.x[i] - a
        bb = h - aa
        return (aa * self.y[i - 1] + bb * self.y[i] -
                (1. / 6.) * aa * bb * ((aa + h) * self.y2[i - 1] + (bb + h) * self.y2[i])) / h


# ---------------------------------------------------------------------------------------------
# Sersic info (src/SBSersic.cpp:301-667)
# ---------------------------------------------------------------------------------------------
_SERSIC = {}


class SersicInfo(object):
    """SersicInfo (src/SBSersic.cpp:288-667); trunc > 0 (in units of r0) for a truncated
    profile: flux fraction gamma_p(2n, trunc^(1/n)) (:332-352), truncated low-k moments and Hankel
    normalisation (:393-424), hankel_trunc values (:453-457), stepk capped at trunc (:304-318)."""

    def __init__(self, n, gsp, trunc=0.):
        self.n = n
        self.gsp = gsp
        self.trunc = float(trunc)
        self.gamma2n = special.gamma(2 * n)
        self.flux_fraction = (special.gammainc(2. * n, self.trunc ** (1. / n)) if self.trunc > 0. else 1.)
        self.b = self._calc_b()
        self.re = self.b ** n
        R = self._missing_flux_radius(gsp.folding_threshold)
        if self.trunc > 0. and self.trunc < R:
            R = self.trunc
        R = max(R, gsp.stepk_minimum_hlr)
        self.stepk = PI / R
        self._build_ft()

    def _missing(self, target):
        twon, gam = 2 * self.n, self.gamma2n
        return lambda z: (1. - special.gammainc(twon, z)) * gam - target

    def _calc_b(self):
        """CalculateB (SBSersic.cpp:627-658) with the profile's flux fraction."""
        n = self.n
        invn = 1. / n
        b1 = 2. * n - 1. / 3.
        b2 = b1 + (8. / 405.) * invn + (46. / 25515.) * invn ** 2 + (131. / 1148175.) * invn ** 3
        return solve_lower_limit(self._missing((1. - 0.5 * self.flux_fraction) * self.gamma2n), b1, b2, 0.)

    def _missing_flux_radius(self, frac):
        n = self.n
        missing = frac * self.gamma2n
        z1 = -math.log(missing)
        if n == 0.5:
            z = z1
        else:
            z = 4. * (n + 1.)
            t = 2. * n - 1.
            z2 = z1 + t * math.log(z) + t / z + t * (2. * n - 3.) / (2. * z * z)
            if z2 > z1 and z2 - z1 < 0.01:
                z2 = z1 + 0.01
            elif z2 < z1 and z2 - z1 > -0.01:
                z2 = z1 - 0.01
            if z1 < 0.:
                z1 = self.b
            z = solve_upper(self._missing(missing), z1, z2)
        return z ** n

    def _build_ft(self):
        n, gsp = self.n, self.gsp
        g2 = special.gamma(2. * n)
        if self.trunc > 0.:
            z = self.trunc ** (1. / n)
            g4, g6, g8 = (special.gammainc(m * n, z) * special.gamma(m * n) for m in (4, 6, 8))
        else:
            g4, g6, g8 = (special.gamma(m * n) for m in (4, 6, 8))
        ff = self.flux_fraction
        self.kd2 = -g4 / (4. * g2) / ff
        self.kd4 = g6 / (64. * g2) / ff
        kd6 = g8 / (2304. * g2) / ff
        kmin = (gsp.kvalue_accuracy / kd6) ** (1. / 6.)
        self.ksq_min = kmin * kmin
        hankel_norm = ff * n * g2
        dlogk = gsp.table_spacing * math.sqrt(math.sqrt(gsp.kvalue_accuracy / 10.))
        f = lambda r: np.exp(-np.power(r, 1. / n))
        n_fit = 10
        fit = []
        sf = skf = sk = sk2 = 0.
        ksq_max = -1.
        maxk = kmin
        found = False
        n_correct = 0
        args, vals = [], []
        a = b = 0.
        logk = math.log(kmin) - 0.001
        i = 0
        while logk < math.log(500.):
            lk = math.log(kmin) - 0.001 + i * dlogk
            k = math.exp(lk)
            ksq = k * k
            if self.trunc > 0.:
                val = hankel_trunc_exact(f, k, self.trunc) / hankel_norm
            else:
                val = hankel_inf(f, k, gsp.integration_relerr, gsp.integration_abserr * hankel_norm) / hankel_norm
            f0 = val * ksq
            args.append(lk)
            vals.append(f0)
            if abs(val) > gsp.maxk_threshold:
                maxk = k
                n_correct = 0
            else:
                found = True
                a = (sf * sk2 - sk * skf) / (n_fit * sk2 - sk * sk)
                b = (n_fit * skf - sk * sf) / (n_fit * sk2 - sk * sk)
                if abs(f0 - (a + b / k)) / ksq < gsp.kvalue_accuracy:
                    n_correct += 1
                else:
                    n_correct = 0
                if n_correct >= 5:
                    ksq_max = ksq
                    break
            inv_k = 1. / k
            if len(fit) == n_fit:
                k_back = math.exp(lk - n_fit * dlogk)
                f_back = fit.pop()
                ikb = 1. / k_back
                sf += f0 - f_back
                skf += f0 * inv_k - f_back * ikb
                sk += inv_k - ikb
                sk2 += inv_k * inv_k - ikb * ikb
            else:
                sf += f0
                skf += f0 * inv_k
                sk += inv_k
                sk2 += inv_k * inv_k
            fit.insert(0, f0)
            i += 1
            logk = math.log(kmin) - 0.001 + i * dlogk
        self.spline = Spline(args, vals)
        if ksq_max <= 0.:
            ksq_max = math.exp(2. * args[-1])
        if found:
            maxk *= math.exp(dlogk)
        else:
            a = (sf * sk2 - sk * skf) / (n_fit * sk2 - sk * sk)
            b = (n_fit * skf - sk * sf) / (n_fit * sk2 - sk * sk)
            maxk = math.sqrt(a / gsp.maxk_threshold)
            for _ in range(3):
                maxk = math.sqrt((a - b / maxk) / gsp.maxk_threshold)
        self.ksq_max = ksq_max
        self.highk_a, self.highk_b = a, b
        self.maxk = maxk

    def kvalue(self, ksq):
        ksq = np.asarray(ksq, float)
        out = np.empty_like(ksq)
        hi = ksq >= self.ksq_max
        lo = ksq < self.ksq_min
        mid = ~hi & ~lo
        out[hi] = (self.highk_a + self.highk_b / np.sqrt(ksq[hi])) / ksq[hi]
        out[lo] = 1. + ksq[lo] * (self.kd2 + ksq[lo] * self.kd4)
        out[mid] = self.spline(0.5 * np.log(ksq[mid])) / ksq[mid]
        return out


def sersic_info(n, gsp=DEFAULT, trunc=0.):
    key = (n, id(gsp), float(trunc))
    if key not in _SERSIC:
        _SERSIC[key] = SersicInfo(n, gsp, trunc)
    return _SERSIC[key]


def sersic_truncated_scale(n, hlr, trunc):
    """SersicTruncatedScale (SBSersic.cpp:700-775): the scale radius that gives a Sersic
    truncated at trunc the half-light radius hlr: b solves gamma_p(2n, b) = gamma_p(2n, x b) / 2
    with x = (trunc / hlr)^(1/n), bracketed between the untruncated b (upper) and an asymptotic
    guess (lower, expanded toward 0); r0 = hlr / b^n."""
    invn = 1. / n
    b = sersic_info(n).b
    t = trunc / hlr
    if t <= math.sqrt(2.):
        raise ValueError("Sersic truncation must be larger than sqrt(2)*half_light_radius.")
    x = t ** invn
    b1 = (math.log(0.5) + (2. * n - 1) * math.log(x)) / (x - 1.)
    if b1 < 1e-3 * b:
        b1 = b / 2.
    twon, gam = 2. * n, special.gamma(2. * n)
    fn = lambda bb: (2. * special.gammainc(twon, bb) - special.gammainc(twon, x * bb)) * gam
    bb = solve_lower_limit(fn, b1, b, 0.)
    return hlr / bb ** n


# ---------------------------------------------------------------------------------------------
# Kolmogorov stepk (src/SBKolmogorov.cpp:338-420)
# ---------------------------------------------------------------------------------------------
_KOLM = {}


def _kolmogorov_info(gsp):
    """KolmogorovInfo (SBKolmogorov.cpp:338-420): the radial table f(r) = hankel(exp(-k^5/3), r)
    / 2 pi at r = 0 (XVAL_ZERO) and r = exp(-3 + i dlogr) until f r^2 / 1.67 < shoot_accuracy / 2 pi,
    its natural spline, and stepk in units of k0."""
    if id(gsp) in _KOLM:
        return _KOLM[id(gsp)]
    dlogr = gsp.table_spacing * math.sqrt(math.sqrt(gsp.xvalue_accuracy / 10.))
    thresh = gsp.shoot_accuracy / (2. * PI)
    f = lambda k: np.exp(-np.power(k, 5. / 3.))
    i = 0
    r1 = F1 = 0.
    rs, vs = [0.], [0.0876786563672346]
    while -3. + i * dlogr < math.log(1.e4):
        r = math.exp(-3. + i * dlogr)
        val = hankel_inf(f, r, gsp.integration_relerr, gsp.integration_abserr) / (2. * PI)
        rs.append(r)
        vs.append(val)
        r1, F1 = r, val
        if val * r * r / 1.67 < thresh:
            break
        i += 1
    nn = 11. / 3.
    R = (2. * PI * F1 * r1 ** nn / ((nn - 2.) * gsp.folding_threshold)) ** (1. / (nn - 2.))
    R = max(R, gsp.stepk_minimum_hlr * 2.992939911888651 * 0.5548101137)
    _KOLM[id(gsp)] = (PI / R, Spline(rs, vs))
    return _KOLM[id(gsp)]


def kolmogorov_stepk_factor(gsp=DEFAULT):
    return _kolmogorov_info(gsp)[0]


def kolmogorov_radial(r, gsp=DEFAULT):
    """KolmogorovInfo::xValue (SBKolmogorov.cpp:114-115): the radial spline, 0 beyond its last node."""
    sp = _kolmogorov_info(gsp)[1]
    r = np.asarray(r, float)
    return np.where(r < sp.x[-1], sp(np.minimum(r, sp.x[-1])), 0.)


# ---------------------------------------------------------------------------------------------
# Clip ranges (src/SBProfile.cpp:508-588)
# ---------------------------------------------------------------------------------------------
def range_1d(m, kmax, ksqmax, kx0, dkx, ky):
    if abs(ky) >= kmax:
        return m, m
    dsq = ksqmax - ky * ky
    if kx0 * kx0 > dsq or (kx0 + m * dkx) ** 2 > dsq:
        d = math.sqrt(dsq)
        i1 = math.ceil((-kx0 - d) / dkx)
        i2 = math.floor((-kx0 + d) / dkx)
        if i1 > i2:
            i1, i2 = i2, i1
        i2 += 1
        if i2 <= 0 or i1 >= m:
            return m, m
        return max(i1, 0), min(i2, m)
    return 0, m


def range_2d(m, kmax, ksqmax, kx0, dkx, ky0, dky):
    if abs(kx0) > kmax or abs(kx0 + m * dkx) > kmax or abs(ky0) > kmax or abs(ky0 + m + dky) > kmax:
        a = dkx * dkx + dky * dky
        b = dkx * kx0 + dky * ky0
        c = kx0 * kx0 + ky0 * ky0 - ksqmax
        d = b * b - a * c
        if d <= 0.:
            return m, m
        d = math.sqrt(d)
        i1 = math.ceil((-b - d) / a)
        i2 = math.floor((-b + d) / a)
        if i1 > i2:
            i1, i2 = i2, i1
        i2 += 1
        if i2 <= 0 or i1 >= m:
            return m, m
        return max(i1, 0), min(i2, m)
    return 0, m


# ---------------------------------------------------------------------------------------------
# Profile tree
# ---------------------------------------------------------------------------------------------
class OObj(object):
    gsp = DEFAULT

    def shear(self, g1, g2):
        gsq = g1 * g1 + g2 * g2
        m = np.array([[1. + g1, g2], [g2, 1. - g1]]) / math.sqrt(1. - gsq)
        return OTransform(self, jac=m)

    def shift(self, dx, dy):
        return OTransform(self, offset=(dx, dy))

    def __mul__(self, s):
        return OTransform(self, flux_ratio=s)

    __rmul__ = __mul__

    def drawK(self, kimage, xmin, ymin, dk, jac):
        """Draw into a complex k-image (numpy, [row, col]) whose corner is (xmin, ymin)."""
        raise NotImplementedError


class OLeaf(OObj):
    axisym_separable = False

    def drawK(self, kimage, xmin, ymin, dk, jac):
        """SBProfile::drawK (SBProfile.cpp:383-425)."""
        nrow, m = kimage.shape
        x0 = xmin * dk
        y0 = ymin * dk
        izero = -xmin if xmin < 0 else 0
        jzero = -ymin if ymin < 0 else 0
        if jac is None or (jac[0, 1] == 0. and jac[1, 0] == 0.):
            mA = 1. if jac is None else jac[0, 0]
            mD = 1. if jac is None else jac[1, 1]
            self.fill_1d(kimage, x0 * mA, dk * mA, izero, y0 * mD, dk * mD, jzero)
        else:
            mA, mB, mC, mD = jac[0, 0], jac[0, 1], jac[1, 0], jac[1, 1]
            self.fill_2d(kimage, mA * x0 + mC * y0, mA * dk, mC * dk, mB * x0 + mD * y0, mD * dk, mB * dk)

    def fill_1d(self, im, kx0, dkx, izero, ky0, dky, jzero):
        if izero != 0 or jzero != 0:
            # FillQuadrant (SBProfile.cpp:434-488)
            n, m = im.shape
            m1, n1 = izero, jzero
            m2, n2 = m - m1 - 1, n - n1 - 1
            q = np.zeros((max(n1, n2) + 1, max(m1, m2) + 1), dtype=im.dtype)
            self.fill_1d(q, kx0 if m1 == 0 else 0., dkx, 0, ky0 if n1 == 0 else 0., dky, 0)
            iq = np.abs(np.arange(m) - m1)
            jq = np.abs(np.arange(n) - n1)
            im[...] = q[jq][:, iq]
            return
        n, m = im.shape
        kx = kx0 + np.arange(m) * dkx
        ky = ky0 + np.arange(n) * dky
        im[...] = self.kv_1d(kx, ky)

    def kv_1d(self, kx, ky):
        KX, KY = np.meshgrid(kx, ky)
        return self.kvalue(KX, KY)

    def fill_2d(self, im, kx0, dkx, dkxy, ky0, dky, dkyx):
        n, m = im.shape
        i = np.arange(m)[None, :]
        j = np.arange(n)[:, None]
        KX = kx0 + j * dkxy + i * dkx
        KY = ky0 + j * dky + i * dkyx
        im[...] = self.kv_2d(KX, KY, kx0, dkx, dkxy, ky0, dky, dkyx, m)

    def kv_2d(self, KX, KY, *grid):
        return self.kvalue(KX, KY)

    def kvalue(self, kx, ky):
        raise NotImplementedError


class OGaussian(OLeaf):
    def __init__(self, sigma, flux=1.):
        self.sigma, self.flux = float(sigma), float(flux)

    def stepk_maxk(self):
        gsp = self.gsp
        maxk = math.sqrt(-2. * math.log(gsp.maxk_threshold)) / self.sigma
        R = max(math.sqrt(-2. * math.log(gsp.folding_threshold)), gsp.stepk_minimum_hlr * 1.1774100225154747)
        return PI / (R * self.sigma), maxk

    def kv_1d(self, kx, ky):
        gx = np.exp(-0.5 * (kx * self.sigma) ** 2)
        gy = np.exp(-0.5 * (ky * self.sigma) ** 2)
        return self.flux * gy[:, None] * gx[None, :]

    def kv_2d(self, KX, KY, *grid):
        ksq = (KX ** 2 + KY ** 2) * self.sigma ** 2
        ksq_max = -2. * math.log(self.gsp.kvalue_accuracy)
        ksq_min = (self.gsp.kvalue_accuracy * 48.) ** (1. / 3.)
        out = self.flux * np.exp(-0.5 * ksq)
        out = np.where(ksq < ksq_min, self.flux * (1. - 0.5 * ksq * (1. - 0.25 * ksq)), out)
        return np.where(ksq > ksq_max, 0., out)


class OExponential(OLeaf):
    def __init__(self, r0, flux=1.):
        self.r0, self.flux = float(r0), float(flux)

    def stepk_maxk(self):
        gsp = self.gsp
        maxk = gsp.maxk_threshold ** (-1. / 3.) / self.r0
        logx = math.log(gsp.folding_threshold)
        R = -logx
        for _ in range(3):
            R = math.log(1. + R) - logx
        R = max(R, gsp.stepk_minimum_hlr * 1.6783469900166605)
        return PI / R / self.r0, maxk

    def _consts(self):
        ksq_max = self.gsp.kvalue_accuracy ** (-1. / 1.5) - 1.
        return ksq_max, math.sqrt(ksq_max)

    def fill_1d(self, im, kx0, dkx, izero, ky0, dky, jzero):
        if izero != 0 or jzero != 0:
            return OLeaf.fill_1d(self, im, kx0, dkx, izero, ky0, dky, jzero)
        n, m = im.shape
        r0 = self.r0
        kx0, dkx, ky0, dky = kx0 * r0, dkx * r0, ky0 * r0, dky * r0
        ksq_max, k_max = self._consts()
        im[...] = 0.
        for j in range(n):
            ky = ky0 + j * dky
            i1, i2 = range_1d(m, k_max, ksq_max, kx0, dkx, ky)
            if i1 == m:
                continue
            kx = kx0 + np.arange(i1, i2) * dkx
            ksqp1 = kx * kx + ky * ky + 1.
            im[j, i1:i2] = self.flux / (ksqp1 * np.sqrt(ksqp1))

    def fill_2d(self, im, kx0, dkx, dkxy, ky0, dky, dkyx):
        n, m = im.shape
        r0 = self.r0
        kx0, dkx, dkxy, ky0, dky, dkyx = (v * r0 for v in (kx0, dkx, dkxy, ky0, dky, dkyx))
        ksq_max, k_max = self._consts()
        im[...] = 0.
        for j in range(n):
            kxj = kx0 + j * dkxy
            kyj = ky0 + j * dky
            i1, i2 = range_2d(m, k_max, ksq_max, kxj, dkx, kyj, dkyx)
            if i1 == m:
                continue
            ii = np.arange(i1, i2)
            kx = kxj + ii * dkx
            ky = kyj + ii * dkyx
            ksqp1 = 1. + kx * kx + ky * ky
            im[j, i1:i2] = self.flux / (ksqp1 * np.sqrt(ksqp1))


class OSersic(OLeaf):
    """Sersic (sersic.py:200-265): trunc > 0 truncates at that radius; without
    flux_untruncated the flux and half-light radius are those of the truncated profile."""

    def __init__(self, n, r0=None, hlr=None, flux=1., trunc=0., flux_untruncated=False):
        self.n, self.flux, self.trunc = float(n), float(flux), float(trunc)
        if r0 is not None:
            self.r0 = float(r0)
        elif self.trunc == 0. or flux_untruncated:
            self.r0 = float(hlr) / sersic_info(self.n, self.gsp).re
        else:
            self.r0 = sersic_truncated_scale(self.n, float(hlr), self.trunc)
        self.info = sersic_info(self.n, self.gsp, self.trunc / self.r0 if self.trunc > 0. else 0.)
        if self.trunc > 0. and flux_untruncated:
            self.flux *= self.info.flux_fraction

    def stepk_maxk(self):
        return self.info.stepk / self.r0, self.info.maxk / self.r0

    def kvalue(self, kx, ky):
        ksq = (kx ** 2 + ky ** 2) * self.r0 ** 2
        return self.flux * self.info.kvalue(ksq)


def moffat_scale_radius_from_hlr(hlr, trunc, beta):
    """MoffatCalculateScaleRadiusFromHLR (SBMoffat.cpp:95-160): analytic without truncation,
    else Brent on 2 f(re) - f(rm) = 0, f(R) = 1 - (1 + R^2/rd^2)^(1-beta), from the untruncated
    value with the upper bracket expanded."""
    r1 = hlr / math.sqrt(0.5 ** (1. / (1. - beta)) - 1.)
    if trunc == 0.:
        return r1
    fn = lambda rd: 2. * (1. - (1. + hlr * hlr / (rd * rd)) ** (1. - beta)) - \
        (1. - (1. + trunc * trunc / (rd * rd)) ** (1. - beta))
    return solve_upper(fn, r1, 2. * r1)


class OMoffat(OLeaf):
    """Moffat (moffat.py:79-125, SBMoffat.cpp:163-345, 498-625); trunc > 0: the FT from a spline
    in k^2 of the truncated Hankel transform (setupFT, :565-625)."""

    def __init__(self, beta, r0=None, fwhm=None, hlr=None, flux=1., trunc=0.):
        self.beta, self.flux, self.trunc = float(beta), float(flux), float(trunc)
        if fwhm is not None:
            r0 = fwhm / (2. * math.sqrt(2. ** (1. / self.beta) - 1.))
        elif hlr is not None:
            r0 = moffat_scale_radius_from_hlr(float(hlr), self.trunc, self.beta)
        self.r0 = float(r0)
        if self.trunc > 0.:
            self._setup_ft()
            return
        kacc = self.gsp.kvalue_accuracy
        b = self.beta
        self.mode, self.nu = 0, b - 1.
        for val, mode, nu in ((1.5, 1, None), (2., 0, 1.), (2.5, 2, None), (3., 0, 2.), (3.5, 3, None),
                              (4., 0, 3.)):
            if abs(b - val) < kacc:
                self.mode = mode
                if nu is not None:
                    self.nu = nu
                break

    def _setup_ft(self):
        gsp, b = self.gsp, self.beta
        self.maxRrD = self.trunc / self.r0
        self.flux_factor = 1. - (1. + self.maxRrD ** 2) ** (1. - b)
        prefactor = 2. * (b - 1.) / self.flux_factor
        dk = gsp.table_spacing * math.sqrt(math.sqrt(gsp.kvalue_accuracy / 10.))
        f = lambda r: (1. + r * r) ** (-b)
        args, vals = [], []
        maxk = 0.
        nbelow = 0
        k = 0.
        while k < 50:
            v = prefactor * hankel_trunc_exact(f, k, self.maxRrD)
            args.append(k * k)
            vals.append(v)
            if abs(v) > gsp.maxk_threshold:
                maxk = k
            nbelow = 0 if abs(v) > gsp.kvalue_accuracy else nbelow + 1
            if nbelow == 5:
                break
            k += dk
        self.ft = Spline(args, vals)
        k1, k2 = maxk, maxk + dk
        if k2 < 50:
            f1, f2 = abs(float(self.ft(k1 * k1))), abs(float(self.ft(k2 * k2)))
            maxk = (k1 * (f2 - gsp.maxk_threshold) + k2 * (gsp.maxk_threshold - f1)) / (f2 - f1)
        self.maxk_rd = maxk

    def kv2(self, k):
        """kV normalised to 1 at k = 0 (SBMoffat.cpp:274-345)."""
        k = np.asarray(k, float)
        if self.mode == 1:
            return np.exp(-k)
        if self.mode == 2:
            return np.exp(-k) * (1. + k)
        if self.mode == 3:
            return np.exp(-k) * (3. + (3. + k) * k) / 3.
        nu = self.nu
        with np.errstate(invalid='ignore', over='ignore'):
            v = special.kv(nu, k) * np.power(k, nu) * 2. ** (1. - nu) / special.gamma(nu)
        return np.where(k == 0., 1., v)

    def stepk_maxk(self):
        gsp = self.gsp
        b, rD = self.beta, self.r0
        if self.trunc > 0.:
            maxk = self.maxk_rd / rD
            maxR = self.maxRrD * rD
            ff = self.flux_factor
        else:
            ksq = solve_upper(lambda q: float(self.kv2(math.sqrt(q))) - gsp.maxk_threshold, 0., 100.)
            maxk = math.sqrt(ksq) / rD
            maxR = math.sqrt(gsp.xvalue_accuracy ** (1. / (1. - b)) - 1.) * rD
            ff = 1.
        if b <= 1.1:
            return PI / maxR, maxk
        R = gsp.folding_threshold ** (0.5 / (1. - b)) * rD
        if R > maxR:
            R = maxR
        hlr = rD * math.sqrt((1. - 0.5 * ff) ** (1. / (1. - b)) - 1.)
        R = max(R, gsp.stepk_minimum_hlr * hlr)
        return PI / R, maxk

    def kvalue(self, kx, ky):
        if self.trunc > 0.:
            ksq = (kx ** 2 + ky ** 2) * self.r0 ** 2
            return self.flux * np.where(ksq > self.ft.x[-1], 0., self.ft(ksq))
        k = np.sqrt(kx ** 2 + ky ** 2) * self.r0
        return self.flux * self.kv2(k)


class OKolmogorov(OLeaf):
    def __init__(self, lam_over_r0=None, fwhm=None, flux=1.):
        if fwhm is not None:
            lam_over_r0 = fwhm / 0.9758634299
        self.lor0, self.flux = float(lam_over_r0), float(flux)
        self.k0 = 2.992939911888651 / self.lor0

    def stepk_maxk(self):
        return kolmogorov_stepk_factor(self.gsp) * self.k0, \
            (-math.log(self.gsp.kvalue_accuracy)) ** 0.6 * self.k0

    def kvalue(self, kx, ky):
        ksq = (kx ** 2 + ky ** 2) / self.k0 ** 2
        return self.flux * np.exp(-np.power(ksq, 5. / 6.))


class OAiry(OLeaf):
    def __init__(self, lam_over_diam, obscuration=0., flux=1.):
        self.lod, self.obs, self.flux = float(lam_over_diam), float(obscuration), float(flux)

    def stepk_maxk(self):
        gsp = self.gsp
        D = 1. / self.lod
        if self.obs == 0.:
            R = 1. / (gsp.folding_threshold * 0.5 * PI * PI)
        else:
            R = 1. / (gsp.folding_threshold * 0.5 * PI * PI * (1. - self.obs))
        R = max(R, gsp.stepk_minimum_hlr * 0.5348321477)
        return PI / R * D, 2. * PI / self.lod

    def kvalue(self, kx, ky):
        D = 1. / self.lod
        t = (kx ** 2 + ky ** 2) / (D * PI) ** 2
        knorm = self.flux / (PI * (1. - self.obs ** 2))
        return knorm * _airy_k(t, self.obs)


def _chord(r, h, rsq, hsq):
    return np.where(r == 0., 0., rsq * np.arcsin(np.clip(h / np.where(r == 0, 1, r), -1, 1)) -
                    h * np.sqrt(np.maximum(rsq - hsq, 0.)))


def _circ_same(r, rsq, tsq):
    hsq = np.maximum(rsq - tsq / 4., 0.)
    h = np.sqrt(hsq)
    out = 2. * _chord(r, h, rsq, hsq)
    out = np.where(tsq == 0., PI * rsq, out)
    return np.where(tsq >= 4. * rsq, 0., out)


def _circ_two(r, s, rsq, ssq, tsq):
    rps = (r + s) ** 2
    rms = (r - s) ** 2
    with np.errstate(divide='ignore', invalid='ignore'):
        hsq = 0.5 * (rsq + ssq) - (tsq * tsq + rps * rms) / (4. * tsq)
    hsq = np.where(np.isfinite(hsq), np.maximum(hsq, 0.), 0.)
    h = np.sqrt(hsq)
    inner = np.where(tsq < rsq - ssq, PI * ssq - _chord(s, h, ssq, hsq) + _chord(r, h, rsq, hsq),
                     _chord(s, h, ssq, hsq) + _chord(r, h, rsq, hsq))
    out = np.where(tsq <= rms, PI * ssq, inner)
    return np.where(tsq >= rps, 0., out)


def _airy_k(t, obs):
    t = np.asarray(t, float)
    if obs == 0.:
        hsq = np.clip(1. - t / 4., 0., 1.)
        h = np.sqrt(hsq)
        out = 2. * (np.arcsin(h) - h * np.sqrt(1. - hsq))
        out = np.where(t == 0., PI, out)
        return np.where(t >= 4., 0., out)
    return _circ_same(1., 1., t) - 2. * _circ_two(1., obs, 1., obs * obs, t) + _circ_same(obs, obs * obs, t)


class OBox(OLeaf):
    def __init__(self, width, height=None, flux=1.):
        self.w = float(width)
        self.h = float(width if height is None else height)
        self.flux = float(flux)

    def stepk_maxk(self):
        return PI / max(self.w, self.h), 2. / (self.gsp.maxk_threshold * min(self.w, self.h))

    @staticmethod
    def _sinc(x):
        x = np.asarray(x, float)
        with np.errstate(invalid='ignore', divide='ignore'):
            v = np.sin(PI * x) / (PI * x)
        return np.where(np.abs(x) < 1.e-4, 1. - (PI * PI / 6.) * x * x, v)

    def kv_1d(self, kx, ky):
        sx = self._sinc(kx * self.w / (2. * PI))
        sy = self._sinc(ky * self.h / (2. * PI))
        return self.flux * sy[:, None] * sx[None, :]

    def kvalue(self, kx, ky):
        return self.flux * self._sinc(kx * self.w / (2. * PI)) * self._sinc(ky * self.h / (2. * PI))


class OConvolve(OObj):
    def __init__(self, *objs):
        self.objs = list(objs)

    def stepk_maxk(self):
        s = [o.stepk_maxk() for o in self.objs]
        inv = 0
        for sk, _ in s:
            inv = inv + sk ** (-2)
        return inv ** (-0.5), min(mk for _, mk in s)

    def drawK(self, kimage, xmin, ymin, dk, jac):
        self.objs[0].drawK(kimage, xmin, ymin, dk, jac)
        tmp = np.empty_like(kimage)
        for o in self.objs[1:]:
            o.drawK(tmp, xmin, ymin, dk, jac)
            kimage *= tmp


class OSum(OObj):
    def __init__(self, *objs):
        self.objs = list(objs)

    def stepk_maxk(self):
        s = [o.stepk_maxk() for o in self.objs]
        return min(sk for sk, _ in s), max(mk for _, mk in s)

    def drawK(self, kimage, xmin, ymin, dk, jac):
        self.objs[0].drawK(kimage, xmin, ymin, dk, jac)
        tmp = np.empty_like(kimage)
        for o in self.objs[1:]:
            o.drawK(tmp, xmin, ymin, dk, jac)
            kimage += tmp


class OTransform(OObj):
    """transform.py:83-604, including the flattening of nested transformations."""

    def __init__(self, obj, jac=None, offset=(0., 0.), flux_ratio=1.):
        self.jac = None if jac is None else np.asarray(jac, float).reshape(2, 2)
        self.dx, self.dy = float(offset[0]), float(offset[1])
        self.flux_ratio = float(flux_ratio)
        if isinstance(obj, OTransform):
            if obj.dx != 0. or obj.dy != 0.:
                if jac is None:
                    dx1, dy1 = obj.dx, obj.dy
                else:
                    dx1 = self.jac[0, 0] * obj.dx + self.jac[0, 1] * obj.dy
                    dy1 = self.jac[1, 0] * obj.dx + self.jac[1, 1] * obj.dy
                self.dx += dx1
                self.dy += dy1
            if jac is None:
                self.jac = obj.jac
            else:
                self.jac = self.jac if obj.jac is None else self.jac.dot(obj.jac)
            self.flux_ratio *= obj.flux_ratio
            self.original = obj.original
        else:
            self.original = obj

    def det(self):
        j = self.jac
        if j is None:
            return 1.
        if j[0, 1] == 0. and j[1, 0] == 0.:
            return j[0, 0] * j[1, 1]
        return j[0, 0] * j[1, 1] - j[0, 1] * j[1, 0]

    def stepk_maxk(self):
        sk, mk = self.original.stepk_maxk()
        if self.jac is None:
            major = minor = 1.
        else:
            j = self.jac
            h1 = math.hypot(j[0, 0] + j[1, 1], j[0, 1] - j[1, 0])
            h2 = math.hypot(j[0, 0] - j[1, 1], j[0, 1] + j[1, 0])
            major, minor = 0.5 * abs(h1 + h2), 0.5 * abs(h1 - h2)
        sk = sk / major
        if self.dx != 0. or self.dy != 0.:
            sk = PI / (PI / sk + math.hypot(self.dx, self.dy))
        return sk, mk / minor

    def drawK(self, kimage, xmin, ymin, dk, jac):
        jac1 = self.jac if jac is None else jac if self.jac is None else jac.dot(self.jac)
        self.original.drawK(kimage, xmin, ymin, dk, jac1)
        fs = abs(self.det()) * self.flux_ratio
        if self.dx != 0. or self.dy != 0.:
            apply_phases(kimage, xmin, ymin, dk, jac, self.dx, self.dy, fs)
        elif abs(fs - 1.) > self.original.gsp.kvalue_accuracy:
            kimage *= fs


def apply_phases(kimage, xmin, ymin, dk, jac, cx, cy, fs):
    """ApplyKImagePhases (SBTransform.cpp:843-883): *= fs exp(-i (kx' cx + ky' cy))."""
    n, m = kimage.shape
    kx = (xmin + np.arange(m))[None, :] * dk
    ky = (ymin + np.arange(n))[:, None] * dk
    if jac is None:
        kxp, kyp = kx, ky
    else:
        kxp = jac[0, 0] * kx + jac[1, 0] * ky
        kyp = jac[0, 1] * kx + jac[1, 1] * ky
    kimage *= fs * np.exp(-1j * (kxp * cx + kyp * cy))


# ---------------------------------------------------------------------------------------------
# InterpolatedImage (interpolatedimage.py:303-685, src/SBInterpolatedImage.cpp,
# src/Interpolant.cpp)
# ---------------------------------------------------------------------------------------------
def lanczos_xval(n, conserve_dc, x):
    """Lanczos::xCalc (Interpolant.cpp:563-716): n sin(pi x) sin(pi x / n) / (pi x)^2 on |x| < n
    (series below 1e-4), divided with conserve_dc by 1 - sum_j 2 K_j (1 - cos(2 pi j x)),
    K_j the kernel's transform at u = j (uCalcRaw)."""
    x = np.abs(np.asarray(x, dtype=float))
    nd = float(n)
    with np.errstate(invalid='ignore', divide='ignore'):
        s = np.sin(PI * x)
        res = nd * s * np.sin(PI * x / nd) / (PI * x) ** 2
    pix = PI * x
    t = pix * pix / 6.
    small = x <= 1.e-4
    s = np.where(small, pix * (1. - t), s)
    res = np.where(small, 1. - t * (1. + 1. / (nd * nd)), res)
    if conserve_dc:
        K = lanczos_k(n)
        c = 1.
        for j in range(1, 6):
            c = c - 2. * K[j] * (1. - np.cos(2. * PI * j * x))
        res = res / c
    return np.where(x >= nd, 0., res)


def interp_xval(name, x):
    """Real-space kernels: Nearest / Linear / Cubic / Quintic (Interpolant.cpp:171-432), Lanczos,
    sinc."""
    lz = _lanczos_name(name)
    if lz is not None:
        return lanczos_xval(lz[0], lz[1], x)
    if name == 'sinc':
        return _sinc(x)
    x = np.abs(np.asarray(x, dtype=float))
    if name == 'nearest':
        return np.where(x > 0.5, 0., 1.)
    if name == 'linear':
        return np.where(x > 1., 0., 1. - x)
    if name == 'cubic':
        return np.where(x < 1., 1. + x * x * (1.5 * x - 2.5),
                        np.where(x < 2., -0.5 * (x - 1.) * (x - 2.) * (x - 2.), 0.))
    if name == 'quintic':
        a = 1. + x * x * x * (-95. / 12. + x * (23. / 2. + x * (-55. / 12.)))
        b = (x - 1.) * (x - 2.) * (-23. / 4. + x * (29. / 2. + x * (-83. / 8. + x * (55. / 24.))))
        c = (x - 2.) * (x - 3.) * (x - 3.) * (-9. / 4. + x * (25. / 12. + x * (-11. / 24.)))
        return np.where(x <= 1., a, np.where(x <= 2., b, np.where(x <= 3., c, 0.)))
    raise ValueError(name)


def _sinc(u):
    """math::sinc (src/math/Sinc.cpp:29-33)."""
    u = np.asarray(u, dtype=float)
    with np.errstate(invalid='ignore', divide='ignore'):
        v = np.sin(PI * u) / (PI * u)
    return np.where(np.abs(u) < 1.e-4, 1. - (PI * PI / 6.) * u * u, v)


def _lanczos_name(name):
    """(n, conserve_dc) of 'lanczosN' / 'lanczosNF' / 'lanczosNT' (interpolant.py:64-110), else None."""
    if not name.startswith('lanczos'):
        return None
    body = name[7:].upper()
    dc = not body.endswith('F')
    return int(body.rstrip('FT')), dc


_LANCZOS = {}


def lanczos_table(n, conserve_dc=True, gsp=DEFAULT):
    """The reference's tabulated Lanczos transform (Lanczos::Lanczos / uCalc / uCalcRaw,
    Interpolant.cpp:719-895): F(u) from sine integrals, with the DC-conserving convolution when
    conserve_dc, at u = 0, du, 2 du, ... (repeated addition, du = table_spacing (kvalue_accuracy
    / 200)^(1/4) / n) while u - uMax < 1/n or u < 1.1, uMax the last u with |F| > kvalue_accuracy;
    returned as (u, F, F'' of the natural cubic spline, uMax)."""
    key = (n, conserve_dc, gsp.table_spacing, gsp.kvalue_accuracy)
    if key in _LANCZOS:
        return _LANCZOS[key]
    nd = float(n)
    si = lambda x: special.sici(x)[0]

    def raw(u):
        vp, vm = nd * (2. * u + 1.), nd * (2. * u - 1.)
        return ((vm - 1.) * si(PI * (vm - 1.)) - (vm + 1.) * si(PI * (vm + 1.)) -
                (vp - 1.) * si(PI * (vp - 1.)) + (vp + 1.) * si(PI * (vp + 1.))) / (2. * PI)

    K = [0.] + [float(raw(float(j))) for j in range(1, 6)]
    C = [1. + 2. * (K[1] * (1. + 3. * K[1] + K[2] + K[3]) + K[2] + K[3] + K[4] + K[5]),
         -K[1] * (1. + 4. * K[1] + K[2] + 2. * K[3]), K[1] * (K[1] - 2. * K[2] + K[3]) - K[2],
         K[1] * (K[1] - 2. * K[3]) - K[3], K[1] * K[3] - K[4], -K[5]]

    def ucalc(u):
        r = raw(u)
        if conserve_dc:
            r = r * C[0] + sum(C[j] * (raw(u + j) + raw(u - j)) for j in range(1, 6))
        return r

    du = gsp.table_spacing * (gsp.kvalue_accuracy / 200.) ** 0.25 / nd
    us, fs = [], []
    u, umax = 0., 0.
    while u - umax < 1. / nd or u < 1.1:
        f = float(ucalc(u))
        us.append(u)
        fs.append(f)
        if abs(f) > gsp.kvalue_accuracy:
            umax = u
        u += du
    x, f = np.array(us), np.array(fs)
    # natural cubic spline: h_{i-1} y2_{i-1} + 2 (h_{i-1} + h_i) y2_i + h_i y2_{i+1} = 6 (slope jumps)
    h = np.diff(x)
    m = len(x)
    ab = np.zeros((3, m - 2))
    ab[0, 1:] = h[1:-1]
    ab[1] = 2. * (h[:-1] + h[1:])
    ab[2, :-1] = h[1:-1]
    rhs = 6. * (np.diff(f[1:]) / h[1:] - np.diff(f[:-1]) / h[:-1])
    from scipy.linalg import solve_banded
    y2 = np.zeros(m)
    y2[1:-1] = solve_banded((1, 1), ab, rhs)
    _LANCZOS[key] = (x, f, y2, umax)
    return _LANCZOS[key]


def lanczos_k(n):
    """K_j = F(j), j = 1..5, of the uncorrected Lanczos transform (Lanczos::Lanczos)."""
    nd = float(n)
    si = lambda x: special.sici(x)[0]

    def raw(u):
        vp, vm = nd * (2. * u + 1.), nd * (2. * u - 1.)
        return ((vm - 1.) * si(PI * (vm - 1.)) - (vm + 1.) * si(PI * (vm + 1.)) -
                (vp - 1.) * si(PI * (vp - 1.)) + (vp + 1.) * si(PI * (vp + 1.))) / (2. * PI)
    return [0.] + [float(raw(float(j))) for j in range(1, 6)]


def lanczos_uval(n, conserve_dc, u, gsp=DEFAULT):
    """Lanczos::uval: the spline of lanczos_table at |u|, 0 above uMax; the interval from the
    equal-spacing lookup of the reference's Table (first node index i >= 1 with u <= u_i)."""
    x, f, y2, umax = lanczos_table(n, conserve_dc, gsp)
    u = np.abs(np.asarray(u, dtype=float))
    m = len(x)
    da = (x[-1] - x[0]) / (m - 1)
    i = np.clip(np.ceil((u - x[0]) / da), 1, m - 1).astype(np.int64)
    hh = x[i] - x[i - 1]
    aa = (x[i] - u) / hh
    bb = 1. - aa
    v = aa * f[i - 1] + bb * f[i] + ((aa ** 3 - aa) * y2[i - 1] + (bb ** 3 - bb) * y2[i]) * hh * hh / 6.
    return np.where(u > umax, 0., v)


def interp_uval(name, u, gsp=DEFAULT):
    """Fourier transforms of the kernels (Interpolant.cpp:176, 251-255, 292-302, 435-461;
    Lanczos from its table, 914-919)."""
    u = np.asarray(u, dtype=float)
    lz = _lanczos_name(name)
    if lz is not None:
        return lanczos_uval(lz[0], lz[1], u, gsp)
    if name == 'delta':
        return np.ones_like(u)
    if name == 'sinc':
        a = np.abs(u)
        return np.where(a > 0.5, 0., np.where(a < 0.5, 1., 0.5))
    s = _sinc(u)
    if name == 'nearest':
        return s
    if name == 'linear':
        return s * s
    c = np.cos(PI * u)
    if name == 'cubic':
        return s * s * s * (3. * s - 2. * c)
    if name == 'quintic':
        ssq = s * s
        piusq = (PI * u) ** 2
        return s * ssq * ssq * (s * (55. - 19. * piusq) + 2. * c * (piusq - 27.))
    raise ValueError(name)


class _XRange(dict):
    """Interpolant::xrange by name; 'lanczosN' has range n."""

    def __missing__(self, name):
        return float(_lanczos_name(name)[0])


INTERP_XRANGE = _XRange({'delta': 0., 'nearest': 0.5, 'linear': 1., 'cubic': 2., 'quintic': 3.,
                         'sinc': 1. / (PI * 1.e-5)})   # sinc: 1 / (pi kvalue_accuracy), default GSParams


def interp_urange(name, kacc, gsp=None):
    """Interpolant::urange (include/galsim/Interpolant.h:237-428, Interpolant.cpp:364, 518;
    Lanczos: its table's uMax)."""
    lz = _lanczos_name(name)
    if lz is not None:
        g = gsp if gsp is not None else OGSParams(kvalue_accuracy=kacc)
        return lanczos_table(lz[0], lz[1], g)[3]
    return {'sinc': lambda: 0.5,
            'delta': lambda: 1. / kacc,
            'nearest': lambda: 1. / (PI * kacc),
            'linear': lambda: math.sqrt(1. / kacc) / PI,
            'cubic': lambda: math.pow((3. * math.sqrt(3.) / 8.) / kacc, 1. / 3.) / PI,
            'quintic': lambda: math.pow((25. * math.sqrt(5.) / 108.) / kacc, 1. / 3.) / PI}[name]()


def interp_krange(name, kacc, gsp=None):
    """Interpolant.krange (interpolant.py:264, 328, 462, 528, 597, 667)."""
    if _lanczos_name(name) is not None:
        return 2. * PI * interp_urange(name, kacc, gsp)
    return {'sinc': PI, 'delta': 2. * PI / kacc, 'nearest': 2. / kacc, 'linear': 2. / kacc ** 0.5,
            'cubic': 1.7320508075688774 / kacc ** (1. / 3.),
            'quintic': 1.6058208066649935 / kacc ** (1. / 3.)}[name]


def size_containing_flux(im, x0, y0, target):
    """CalculateSizeContainingFlux (SBInterpolatedImage.cpp:1084-1110) on an image array
    whose pixel [0, 0] sits at centred coordinates (x0, y0)."""
    ny, nx = im.shape
    at = lambda x, y: im[y - y0, x - x0]
    p = 1. if target > 0. else -1.
    dmax = min((nx - 1) // 2, (ny - 1) // 2)
    flux = at(0, 0)
    d = 1
    while d <= dmax:
        for x in range(-d, d):
            flux += at(x, -d)
            flux += at(d, x)
            flux += at(-x, d)
            flux += at(-d, -x)
        if p * flux >= p * target:
            break
        d += 1
    return d + 0.5


class OInterpolatedImageLeaf(OLeaf):
    """SBInterpolatedImage in image units: the k interpolant over the padded image's DFT times
    the x interpolant's transform (SBInterpolatedImage.cpp:385-448 kValue, 767-936 separable
    fill with its integer shortcut, 938-1000 general fill)."""

    def __init__(self, xim, x_interp='quintic', k_interp='quintic', gsp=DEFAULT):
        N = xim.shape[0]
        self.N = N
        # K(p, q) = sum I(X, Y) exp(-2 pi i (p X + q Y) / N), X = column - N/2 (checkK / rfft)
        self.K = np.fft.fft2(np.fft.ifftshift(xim))
        self.xi, self.ki = x_interp, k_interp
        self.xr = INTERP_XRANGE[k_interp]
        self.kscale = (N // 2) / PI
        self.uscale = 1. / (2. * PI)
        self.maxk1 = interp_urange(x_interp, gsp.kvalue_accuracy, gsp) / self.uscale
        self.gsp = gsp

    def _taps(self, s, shortcut):
        """Tap positions p[..., t] and weights w[..., t] for sample positions s."""
        nt = int(2 * self.xr) + 1
        p1 = np.ceil(s - self.xr)
        t = np.arange(nt)
        p = p1[..., None] + t
        w = interp_xval(self.ki, p - s[..., None])
        if shortcut:
            small = 10. * np.finfo(float).eps
            fl = np.floor(s + 0.01)
            on = np.abs(s - fl) < small * (np.abs(s) + 1.)
            p = np.where(on[..., None], fl[..., None] + t, p)
            w1 = interp_xval(self.ki, fl - s)
            w = np.where(on[..., None], np.where(t == 0, w1[..., None], 0.), w)
        return p.astype(np.int64), w

    def kv(self, KX, KY, shortcut):
        KX = np.asarray(KX, float)
        KY = np.asarray(KY, float)
        px, wx = self._taps(KX * self.kscale, shortcut)
        py, wy = self._taps(KY * self.kscale, shortcut)
        N = self.N
        vals = self.K[(py[..., :, None] % N), (px[..., None, :] % N)]
        s = np.einsum('...ba,...a,...b->...', vals, wx, wy)
        fac = interp_uval(self.xi, KX * self.uscale, self.gsp) * interp_uval(self.xi, KY * self.uscale, self.gsp)
        out = fac * s
        return np.where((np.abs(KX) > self.maxk1) | (np.abs(KY) > self.maxk1), 0., out)

    def fill_1d(self, im, kx0, dkx, izero, ky0, dky, jzero):
        n, m = im.shape
        kx = kx0 + np.arange(m) * dkx
        ky = ky0 + np.arange(n) * dky
        KX, KY = np.meshgrid(kx, ky)
        im[...] = self.kv(KX, KY, True)

    def kv_2d(self, KX, KY, *grid):
        return self.kv(KX, KY, False)

    def kvalue(self, kx, ky):
        return self.kv(kx, ky, True)

    def max_k(self, flux, max_maxk=0.):
        """calculateMaxK (SBInterpolatedImage.cpp:1146-1213), image units."""
        N, No2 = self.N, self.N // 2
        dk = PI / No2
        thresh = (self.gsp.maxk_threshold * flux) ** 2
        if max_maxk == 0.:
            max_maxk = self.maxk1
        max_ix = min(int(math.ceil(max_maxk / dk)), No2)
        nrm = lambda p, q: abs(self.K[q % N, p % N]) ** 2
        maxk_ix = 0.
        below = 0
        for ix in range(max_ix + 1):
            for iy in range(ix + 1):
                v = nrm(iy, -ix)
                if v <= thresh and iy != ix and ix != No2:
                    v = nrm(iy, ix)
                if v <= thresh and iy > 0:
                    v = nrm(ix, -iy)
                if v <= thresh and ix > 0 and iy != No2:
                    v = nrm(ix, iy)
                if v > thresh:
                    maxk_ix = ix
                    below = 0
                    break
            below += 1
            if below == 5:
                break
        return (maxk_ix + 1.) * dk


class OInterpolatedImage(OObj):
    """InterpolatedImage(image, scale=..., ...) (interpolatedimage.py:303-400, 447-566,
    590-685): the padded frame (with Gaussian noise padding from a BaseDeviate seed), flux,
    stepk / maxk in world units, and the world profile
    Transform(Shift(SBInterpolatedImage, -offset), scale, flux_ratio)."""

    def __init__(self, array, scale, x_interp='quintic', k_interp='quintic', flux=None,
                 normalization='flux', pad_factor=4., offset=(0., 0.), use_true_center=True,
                 calculate_stepk=True, calculate_maxk=True, pad_image=None, force_stepk=0.,
                 force_maxk=0., noise_pad_size=0., noise_pad=0., rng_seed=None, gsp=DEFAULT):
        arr = np.asarray(array, dtype=float)
        ny, nx = arr.shape
        # setCenter(0, 0): pixel [0, 0] at (-(nx // 2), -(ny // 2))
        x0, y0 = -(nx // 2), -(ny // 2)
        dx, dy = float(offset[0]), float(offset[1])
        if use_true_center:
            if nx % 2 == 0:
                dx -= 0.5
            if ny % 2 == 0:
                dy -= 0.5
        pad = max(nx, ny)
        if pad_factor > 1.:
            pad = int(math.ceil(pad_factor * pad))
        npad = 0
        if noise_pad:
            # Gaussian noise padding (interpolatedimage.py:463-471, 521-566): a square of
            # good_fft_size(ceil(size / scale)) pixels centred on (0, 0)
            npad = good_fft_size(int(math.ceil(noise_pad_size / scale)))
            pad = max(pad, npad)
        if pad_image is not None:
            pad = max(pad, *np.shape(pad_image))
        N = good_fft_size(pad)
        xim = np.zeros((N, N))
        nz = np.zeros((N, N), dtype=bool)
        if npad:
            noise = gaussian_noise(np.zeros((npad, npad)), base_deviate(rng_seed), math.sqrt(noise_pad))
            h = npad // 2
            xim[N // 2 - h:N // 2 - h + npad, N // 2 - h:N // 2 - h + npad] = noise
            nz[N // 2 - h:N // 2 - h + npad, N // 2 - h:N // 2 - h + npad] = True
        if pad_image is not None:
            pim = np.asarray(pad_image, dtype=float)
            pny, pnx = pim.shape
            px0, py0 = -(pnx // 2), -(pny // 2)
            xim[py0 + N // 2:py0 + N // 2 + pny, px0 + N // 2:px0 + N // 2 + pnx] = pim
            nz[py0 + N // 2:py0 + N // 2 + pny, px0 + N // 2:px0 + N // 2 + pnx] = True
        xim[y0 + N // 2:y0 + N // 2 + ny, x0 + N // 2:x0 + N // 2 + nx] = arr
        nz[y0 + N // 2:y0 + N // 2 + ny, x0 + N // 2:x0 + N // 2 + nx] = True
        self.N = N
        self.leaf = OInterpolatedImageLeaf(xim, x_interp, k_interp, gsp)
        image_flux = float(np.sum(arr, dtype=np.float64))
        # getFlux of the nonzero image: the bounding box of image and pad image
        rows, cols = np.nonzero(nz)
        # for real-space drawing: the padded image and its nonzero bounds in frame coordinates
        self.leaf.xim = xim
        self.leaf.nzb = (cols.min() - N // 2, cols.max() - N // 2, rows.min() - N // 2, rows.max() - N // 2)
        nz_flux = float(np.sum(xim[rows.min():rows.max() + 1, cols.min():cols.max() + 1]))
        if flux is None:
            flux = image_flux * (scale * scale if normalization.lower() in ('sb', 'surface brightness')
                                 else 1.)
        self.flux = flux
        if force_stepk > 0.:
            self.stepk = force_stepk
        else:
            if calculate_stepk:
                R = size_containing_flux(arr, x0, y0, (1. - gsp.folding_threshold) * image_flux)
            else:
                R = max(nx, ny) / 2. - 0.5
            self.stepk = PI / (math.hypot(R, INTERP_XRANGE[x_interp]) * scale)
        if force_maxk > 0.:
            self.maxk = force_maxk
        elif calculate_maxk:
            mm = 0. if calculate_maxk is True else float(calculate_maxk)
            self.maxk = self.leaf.max_k(nz_flux, mm) / scale
        else:
            self.maxk = interp_krange(x_interp, gsp.kvalue_accuracy, gsp) / scale
        prof = self.leaf
        if dx != 0. or dy != 0.:
            prof = OTransform(prof, offset=(-dx, -dy))
        fr = flux / image_flux if flux != image_flux else 1.
        jac = None if scale == 1. else [[scale, 0.], [0., scale]]
        self.inner = OTransform(prof, jac=jac, flux_ratio=(1. / scale) ** 2 * fr)

    def stepk_maxk(self):
        return self.stepk, self.maxk

    def drawK(self, kimage, xmin, ymin, dk, jac):
        self.inner.drawK(kimage, xmin, ymin, dk, jac)


# ---------------------------------------------------------------------------------------------
# Image-level steps
# ---------------------------------------------------------------------------------------------
def good_fft_size(n):
    """goodFFTSize (src/Image.cpp:1141-1153)."""
    if n <= 2:
        return 2
    insize = (1. - 1.e-5) * n
    log2n = math.log(2.) * math.ceil(math.log(insize) / math.log(2.))
    log2n3 = math.log(3.) + math.log(2.) * math.ceil((math.log(insize) - math.log(3.)) / math.log(2.))
    log2n3 = max(log2n3, math.log(6.))
    return int(math.ceil(math.exp(min(log2n, log2n3)) - 1.e-5))


def wrap_hermx(im, ky_min, N):
    """wrapImage(hermx=True) of a complex k-image whose rows are ky = ky_min.. and columns
    kx = 0..m-1, onto rows -N/2..N/2-1 and columns 0..N/2; the pointer walk of
    src/Image.cpp:482-576 and 578-715 restated.  Modifies im in place; returns the subimage."""
    n, m = im.shape
    mwrap = N // 2 + 1
    j1 = -N // 2 - ky_min
    j2 = j1 + N
    nwrap = N
    cj = np.conj
    mid = (n - 1) // 2
    for j in range(mid):
        A = im[j]
        B = im[n - 1 - j]
        p1 = p1w = p2 = p2w = mwrap - 1
        i = mwrap - 1
        while True:
            temp = A[p1]
            A[p1w] += cj(B[p2])
            B[p2w] += cj(temp)
            p1 += 1; p2 += 1; p1w -= 1; p2w -= 1; i += 1
            for _ in range(min(m - i, mwrap - 2)):
                A[p1w] += cj(B[p2])
                B[p2w] += cj(A[p1])
                p1w -= 1; p2w -= 1; p1 += 1; p2 += 1; i += 1
            if i == m:
                break
            A[p1w] += cj(B[p2])
            B[p2w] += cj(A[p1])
            for _ in range(min(m - i, mwrap - 1)):
                A[p1w] += A[p1]
                B[p2w] += B[p2]
                p1w += 1; p2w += 1; p1 += 1; p2 += 1; i += 1
            if i == m:
                break
            A[p1w] += A[p1]
            B[p2w] += B[p2]
    R = im[mid]
    p = pw = mwrap - 1
    i = mwrap - 1
    while True:
        for _ in range(min(m - i, mwrap - 1)):
            R[pw] += cj(R[p])
            pw -= 1; p += 1; i += 1
        if i == m:
            break
        R[pw] += cj(R[p])
        for _ in range(min(m - i, mwrap - 1)):
            R[pw] += R[p]
            pw += 1; p += 1; i += 1
        if i == m:
            break
        R[pw] += R[p]
    # rows (non-Hermitian y direction), src/Image.cpp:690-712
    jj = j2 - (j2 % nwrap)
    if jj == j2:
        jj = j1
    j = 0
    while j < n:
        if j == j1:
            j = j2
        for _ in range(min(n - j, j2 - jj)):
            im[jj] += im[j]
            j += 1
            jj += 1
        jj = j1
    return im[j1:j2, 0:mwrap]


def irfft_shifted(kw, N):
    """irfft(kimage, out, shift_in=True, shift_out=True) (src/Image.cpp:815-912): input rows
    ky = -N/2..N/2-1, columns kx = 0..N/2; output real image [y, x] for x, y = -N/2..N/2-1."""
    K = np.concatenate([kw[N // 2:], kw[:N // 2]], axis=0)          # shift_in: ky = 0 first
    r = np.arange(N)[:, None]
    i = np.arange(N // 2 + 1)[None, :]
    K = K * np.where((r + i) % 2 == 0, 1., -1.)                      # shift_out
    return np.fft.irfft2(K, s=(N, N))                                # includes 1/(Nx Ny)


def size_for_image(obj, bounds, gsp=DEFAULT):
    """drawFFT_makeKImage sizing (gsobject.py:1900-1963) for an image view with the given
    (centred) bounds (xmin, xmax, ymin, ymax)."""
    stepk, maxk = obj.stepk_maxk()
    Nd = 2. * PI / stepk
    N = int(math.ceil(Nd * (1. - 1.e-12)))
    N = 2 * ((N + 1) // 2)
    image_N = max(max(abs(v) for v in bounds) * 2, max(bounds[3] - bounds[2] + 1, bounds[1] - bounds[0] + 1))
    N = max(N, image_N)
    N = good_fft_size(N)
    N = max(N, gsp.minimum_fft_size)
    dk = 2. * PI / N
    if N * dk / 2 > maxk:
        Nk = N
    else:
        Nk = int(np.ceil(maxk / dk)) * 2
    return N, Nk


def draw_fft(obj, bounds, gsp=DEFAULT):
    """drawFFT (gsobject.py:2014-2045) into a float64 image with centred bounds
    (xmin, xmax, ymin, ymax).  Returns (array[ny, nx], added_flux, N, Nk)."""
    N, Nk = size_for_image(obj, bounds, gsp)
    dk = 2. * PI / N
    kim = np.zeros((Nk + 1, Nk // 2 + 1), dtype=np.complex128)
    obj.drawK(kim, 0, -Nk // 2, dk, None)
    kw = wrap_hermx(kim, -Nk // 2, N)
    real = irfft_shifted(np.array(kw), N)
    xmin, xmax, ymin, ymax = bounds
    sub = real[ymin + N // 2:ymax + N // 2 + 1, xmin + N // 2:xmax + N // 2 + 1]
    return sub.copy(), float(sub.sum(dtype=float)), N, Nk


def draw_image(prof, nx, ny, scale, offset=(0., 0.), method='fft', use_true_center=True,
               gsp=DEFAULT):
    """drawImage(nx=, ny=, scale=, method='fft' | 'no_pixel', offset=) (gsobject.py:1283-1844)
    for a world-coordinate profile.  Returns (array, added_flux, N, Nk)."""
    dx, dy = float(offset[0]), float(offset[1])
    if use_true_center:
        if nx % 2 == 0:
            dx -= 0.5
        if ny % 2 == 0:
            dy -= 0.5
    inv = 1. / scale
    jac = None if scale == 1. else np.array([[inv, 0.], [0., inv]])
    img_prof = OTransform(prof, jac=jac, offset=(dx, dy), flux_ratio=scale ** 2)
    if method == 'fft':
        img_prof = OConvolve(img_prof, OBox(1.0))
    # bounds 1..nx, 1..ny shifted by -center
    cx = 1 + nx // 2
    cy = 1 + ny // 2
    bounds = (1 - cx, nx - cx, 1 - cy, ny - cy)
    return draw_fft(img_prof, bounds, gsp)


# ---------------------------------------------------------------------------------------------
# Real-space drawing (drawReal: gsobject.py:1846-1898; transform.py:571-583; sum.py:304-310;
# SBProfile::draw, SBProfile.cpp:305-383; the profiles' xValue / fillXImage)
# ---------------------------------------------------------------------------------------------
def _leaf_xvalue(leaf, u, v):
    gsp = leaf.gsp
    if isinstance(leaf, OGaussian):                       # SBGaussian.cpp:57-69, 99-103
        iss = (1. / leaf.sigma) ** 2
        return leaf.flux * iss / (2. * PI) * np.exp(-0.5 * (u * u + v * v) * iss)
    if isinstance(leaf, OExponential):                    # SBExponential.cpp:67-82, 99-103
        ir = 1. / leaf.r0
        return (leaf.flux / (2. * PI)) * (ir * ir) * np.exp(-np.sqrt(u * u + v * v) * ir)
    if isinstance(leaf, OSersic):                         # SBSersic.cpp:71-96, 354-361
        n, r0 = leaf.n, leaf.r0
        ff = leaf.info.flux_fraction if leaf.trunc > 0. else 1.
        ir2 = (1. / r0) ** 2
        xnorm = leaf.flux * (1. / (2. * PI * n * math.gamma(2. * n) * ff)) * ir2
        rsq = (u * u + v * v) * ir2
        val = xnorm * np.exp(-np.power(rsq, 1. / (2. * n)))
        if leaf.trunc > 0.:
            val = np.where(rsq > (leaf.trunc / r0) ** 2, 0., val)
        return val
    if isinstance(leaf, OMoffat):                         # SBMoffat.cpp:163-203, 256-261
        b, rD = leaf.beta, leaf.r0
        if leaf.trunc > 0.:
            maxRrD = leaf.trunc / rD
            ff = 1. - (1. + maxRrD * maxRrD) ** (1. - b)
        else:
            ff = 1.
            maxRrD = math.sqrt(gsp.xvalue_accuracy ** (1. / (1. - b)) - 1.)
        norm = leaf.flux * (b - 1.) / (PI * ff * rD * rD)
        rsq = (u * u + v * v) / (rD * rD)
        return np.where(rsq > maxRrD * maxRrD, 0., norm * np.power(1. + rsq, -b))
    if isinstance(leaf, OKolmogorov):                     # SBKolmogorov.cpp:85-115
        k0 = leaf.k0
        return leaf.flux * k0 * k0 * kolmogorov_radial(np.sqrt(u * u + v * v) * k0, gsp)
    if isinstance(leaf, OAiry):                           # SBAiry.cpp:66-117, 392-428
        D = 1. / leaf.lod
        obs = leaf.obs
        nu = np.sqrt(u * u + v * v) * D * PI
        thresh = math.sqrt(8. * gsp.xvalue_accuracy)
        with np.errstate(invalid='ignore', divide='ignore'):
            if obs == 0.:
                x = np.where(nu < thresh, 0.5, special.j1(nu) / nu)
                norm = PI
            else:
                x = np.where(nu < thresh, 0.5 * (1. - obs * obs),
                             (special.j1(nu) - obs * special.j1(obs * nu)) / nu)
                norm = PI / (1. - obs * obs)
        return leaf.flux * D * D * (x * x * norm)
    raise NotImplementedError(type(leaf).__name__)


def ii_xvalue(leaf, u, v):
    """SBInterpolatedImage::xValue (SBInterpolatedImage.cpp:167-215) at arrays of positions:
    the x interpolant's taps within its half-width (one tap along an axis at an integer to
    10 eps), clipped to the nonzero bounds, summed over the padded image."""
    small = 10. * np.finfo(float).eps
    xr = INTERP_XRANGE[leaf.xi] if leaf.xi != 'sinc' else 1. / (PI * leaf.gsp.kvalue_accuracy)
    bx0, bx1, by0, by1 = leaf.nzb
    N = leaf.N
    out = np.zeros(np.broadcast(u, v).shape)
    uu, vv = np.broadcast_arrays(u, v)
    for idx in np.ndindex(out.shape):
        x, y = float(uu[idx]), float(vv[idx])
        fx, fy = math.floor(x + 0.01), math.floor(y + 0.01)
        if abs(x - fx) < small * (abs(x) + 1.):
            p1 = p2 = int(fx)
        else:
            p1, p2 = int(math.ceil(x - xr)), int(math.floor(x + xr))
        if abs(y - fy) < small * (abs(y) + 1.):
            q1 = q2 = int(fy)
        else:
            q1, q2 = int(math.ceil(y - xr)), int(math.floor(y + xr))
        if p2 < bx0 or p1 > bx1 or q2 < by0 or q1 > by1:
            continue
        p1, p2, q1, q2 = max(p1, bx0), min(p2, bx1), max(q1, by0), min(q2, by1)
        wx = interp_xval(leaf.xi, np.arange(p1, p2 + 1) - x)
        wy = interp_xval(leaf.xi, np.arange(q1, q2 + 1) - y)
        sub = leaf.xim[q1 + N // 2:q2 + N // 2 + 1, p1 + N // 2:p2 + N // 2 + 1]
        out[idx] = float(wy @ (sub @ wx))
    return out


def draw_real_leaf(leaf, nx, ny, xmin, ymin, jac, xoff, yoff, flux_ratio):
    """SBProfile::draw with imscale 1 for one leaf: the image positions xmin + i, ymin + j."""
    x0, y0 = xmin - xoff, ymin - yoff
    i = np.arange(nx)[None, :].astype(float)
    j = np.arange(ny)[:, None].astype(float)
    amp = flux_ratio
    if jac is None:
        mode, u0, du, duy, v0, dv, dvx = 0, x0, 1., 0., y0, 1., 0.
    elif jac[0, 1] == 0. and jac[1, 0] == 0.:
        xs, ys = 1. / jac[0, 0], 1. / jac[1, 1]
        mode, u0, du, duy, v0, dv, dvx = 1, x0 * xs, xs, 0., y0 * ys, ys, 0.
        amp *= abs(xs * ys)
    else:
        A, B, C, D = jac[0, 0], jac[0, 1], jac[1, 0], jac[1, 1]
        invdet = 1. / (A * D - B * C)
        mode = 2
        u0, v0 = (D * x0 - B * y0) * invdet, (-C * x0 + A * y0) * invdet
        du, duy, dv, dvx = D * invdet, -B * invdet, A * invdet, -C * invdet
        amp *= abs(invdet)
    if isinstance(leaf, OBox):                            # SBBox.cpp:79-150
        norm = leaf.flux / (leaf.w * leaf.h)
        if mode <= 1:
            bx0, by0 = u0 / du, v0 / dv
            wo2, ho2 = 0.5 * leaf.w / abs(du), 0.5 * leaf.h / abs(dv)
            inside = ((i >= np.ceil(-wo2 - bx0)) & (i < np.ceil(wo2 - bx0)) &
                      (j >= np.ceil(-ho2 - by0)) & (j < np.ceil(ho2 - by0)))
        else:
            x = u0 + i * du + j * duy
            y = v0 + j * dv + i * dvx
            inside = (np.abs(x) < 0.5 * leaf.w) & (np.abs(y) < 0.5 * leaf.h)
        return amp * np.where(inside, norm, 0.)
    u = u0 + i * du + j * duy
    v = v0 + j * dv + i * dvx
    if isinstance(leaf, OInterpolatedImageLeaf):
        return amp * ii_xvalue(leaf, u, v)
    return amp * _leaf_xvalue(leaf, u, v)


def draw_real(obj, nx, ny, xmin, ymin, jac=None, offset=(0., 0.), flux_scaling=1.):
    """The _drawReal walk (transform.py:571-583, sum.py:304-310) summed in FP64."""
    if isinstance(obj, OTransform):
        dx, dy = offset
        if obj.dx != 0. or obj.dy != 0.:
            if jac is not None:
                x1 = jac[0, 0] * obj.dx + jac[0, 1] * obj.dy
                y1 = jac[1, 0] * obj.dx + jac[1, 1] * obj.dy
            else:
                x1, y1 = obj.dx, obj.dy
            dx += x1
            dy += y1
        flux_scaling *= abs(obj.det()) * obj.flux_ratio
        jac = obj.jac if jac is None else jac if obj.jac is None else jac.dot(obj.jac)
        return draw_real(obj.original, nx, ny, xmin, ymin, jac, (dx, dy), flux_scaling)
    if isinstance(obj, OSum):
        return sum(draw_real(o, nx, ny, xmin, ymin, jac, offset, flux_scaling) for o in obj.objs)
    if isinstance(obj, OInterpolatedImage):
        return draw_real(obj.inner, nx, ny, xmin, ymin, jac, offset, flux_scaling)
    return draw_real_leaf(obj, nx, ny, xmin, ymin, jac, offset[0], offset[1], flux_scaling)


def draw_image_real(prof, nx, ny, scale, offset=(0., 0.), method='no_pixel', use_true_center=True):
    """drawImage(method='no_pixel' | 'sb') of a profile analytic in real space (gsobject.py:
    1647-1811 with drawReal).  Returns (array, added_flux)."""
    dx, dy = float(offset[0]), float(offset[1])
    if use_true_center:
        if nx % 2 == 0:
            dx -= 0.5
        if ny % 2 == 0:
            dy -= 0.5
    inv = 1. / scale
    jac = None if scale == 1. else np.array([[inv, 0.], [0., inv]])
    fr = scale ** 2 / (scale * scale if method == 'sb' else 1.)
    img_prof = OTransform(prof, jac=jac, offset=(dx, dy), flux_ratio=fr)
    xmin, ymin = -(nx // 2), -(ny // 2)
    arr = draw_real(img_prof, nx, ny, xmin, ymin)
    flux_scale = 1. / (scale * scale) if method == 'sb' else 1.
    return arr, float(arr.sum()) / flux_scale


def draw_kimage(obj, nkx, nky, kxmin, kymin, dk):
    """_drawKImage on a grid with corner (kxmin, kymin) (gsobject.py:2575-2582)."""
    kim = np.zeros((nky, nkx), dtype=np.complex128)
    obj.drawK(kim, kxmin, kymin, dk, None)
    return kim


# ---------------------------------------------------------------------------------------------
# Noise (galsim/noise.py, galsim/random.py, src/Random.cpp with the Boost.Random 1.48 engines
# and distributions it vendors): pure-Python restatement for small images.
# ---------------------------------------------------------------------------------------------
class OMersenneTwister(object):
    """Mersenne Twister (Matsumoto & Nishimura 1998) with the init_genrand seeding of
    2002 (mersenne_twister.hpp:154-185, 430-478)."""

    def __init__(self, w, n, m, r, a, u, s, b, t, c, l, f, seed):
        self.n, self.m, self.r, self.a = n, m, r, a
        self.u, self.s, self.b, self.t, self.c, self.l = u, s, b, t, c, l
        mask = 0xffffffff
        x = [0] * n
        x[0] = seed & mask
        for i in range(1, n):
            x[i] = (f * (x[i - 1] ^ (x[i - 1] >> (w - 2))) + i) & mask
        if (x[0] & ((mask << r) & mask)) == 0 and all(v == 0 for v in x[1:]):
            x[0] = 1 << (w - 1)
        self.x = x
        self.i = n

    def _twist(self):
        n, m, x = self.n, self.m, self.x
        upper = (0xffffffff << self.r) & 0xffffffff
        lower = (~upper) & 0xffffffff
        for j in range(n):
            y = (x[j] & upper) | (x[(j + 1) % n] & lower)
            x[j] = x[(j + m) % n] ^ (y >> 1) ^ ((x[(j + 1) % n] & 1) * self.a)
        self.i = 0

    def __call__(self):
        if self.i == self.n:
            self._twist()
        z = self.x[self.i]
        self.i += 1
        z ^= (z >> self.u)
        z ^= (z << self.s) & self.b
        z ^= (z << self.t) & self.c
        z ^= (z >> self.l)
        return z & 0xffffffff


def mt19937(seed):
    return OMersenneTwister(32, 624, 397, 31, 0x9908b0df, 11, 7, 0x9d2c5680, 15, 0xefc60000, 18,
                            1812433253, seed)


def mt11213b(seed):
    return OMersenneTwister(32, 351, 175, 19, 0xccab8ee7, 11, 7, 0x31b6ab00, 15, 0xffe50000, 17,
                            1812433253, seed)


def base_deviate(seed):
    """BaseDeviate(seed) (Random.cpp:156-191): the seed goes through 2 discarded draws of an
    mt11213b, whose third draw seeds the mt19937 used for everything."""
    alt = mt11213b(int(seed) & 0xffffffff)
    alt()
    alt()
    return mt19937(alt())


def uniform01(rng):
    """boost uniform_01 on a 32-bit engine: one draw times 2^-32."""
    return rng() * (1. / 4294967296.)


class ONormal(object):
    """boost 1.48 normal_distribution: Box-Muller pairs, cos first (normal_distribution.hpp:153-175)."""

    def __init__(self, mean=0., sigma=1.):
        self.mean, self.sigma = mean, sigma
        self.valid = False

    def reset(self):
        self.valid = False

    def __call__(self, rng):
        if not self.valid:
            self.r1 = uniform01(rng)
            self.r2 = uniform01(rng)
            self.rho = math.sqrt(-2. * math.log(1. - self.r2))
            self.valid = True
            return self.rho * math.cos(2. * PI * self.r1) * self.sigma + self.mean
        self.valid = False
        return self.rho * math.sin(2. * PI * self.r1) * self.sigma + self.mean


_LOG_FACT = [math.lgamma(k + 1.) for k in range(10)]


def poisson_draw(mean, rng):
    """boost 1.48 poisson_distribution: inversion below mean 10, otherwise the PTRD transformed
    rejection of Hoermann (1993) (poisson_distribution.hpp)."""
    if mean < 10:
        p = math.exp(-mean)
        x = 0
        u = uniform01(rng)
        while u > p:
            u = u - p
            x += 1
            p = mean * p / x
        return x
    smu = math.sqrt(mean)
    b = 0.931 + 2.53 * smu
    a = -0.059 + 0.02483 * b
    inv_alpha = 1.1239 + 1.1328 / (b - 3.4)
    v_r = 0.9277 - 3.6224 / (b - 2)
    while True:
        v = uniform01(rng)
        if v <= 0.86 * v_r:
            u = v / v_r - 0.43
            return int(math.floor((2 * a / (0.5 - abs(u)) + b) * u + mean + 0.445))
        if v >= v_r:
            u = uniform01(rng) - 0.5
        else:
            u = v / v_r - 0.93
            u = (-0.5 if u < 0 else 0.5) - u
            v = uniform01(rng) * v_r
        us = 0.5 - abs(u)
        if us < 0.013 and v > us:
            continue
        k = math.floor((2 * a / us + b) * u + mean + 0.445)
        v = v * inv_alpha / (a / (us * us) + b)
        if k >= 10:
            if math.log(v * smu) <= ((k + 0.5) * math.log(mean / k) - mean - 0.91893853320467267 + k
                                     - (1 / 12. - (1 / 360. - 1 / (1260. * k * k)) / (k * k)) / k):
                return int(k)
        elif k >= 0:
            if math.log(v) <= k * math.log(mean) - mean - _LOG_FACT[int(k)]:
                return int(k)


class OPoissonDeviate(object):
    """PoissonDeviate with the mean switching of Random.cpp:498-540: Gaussian above 2^30."""

    def __init__(self, rng):
        self.rng = rng
        self.mean = -1.
        self.gd = None
        self.set_mean(1.)

    def set_mean(self, mean):
        if mean != self.mean:
            self.mean = mean
            if mean > float(1 << 30) or mean == 0.:
                if self.gd is None:
                    self.gd = ONormal(mean, math.sqrt(mean))
                else:
                    self.gd.mean, self.gd.sigma = mean, math.sqrt(mean)
                self.use_gd = True
            else:
                self.gd = None
                self.use_gd = False

    def __call__(self):
        return self.gd(self.rng) if self.use_gd else float(poisson_draw(self.mean, self.rng))


def weibull_draw(rng, a, b):
    """boost 1.48 weibull_distribution: b (-ln(1 - u))^(1/a)."""
    return b * math.pow(-math.log(1. - uniform01(rng)), 1. / a)


def gamma_draw(rng, alpha, beta):
    """boost 1.48 gamma_distribution: exponential (alpha = 1), tangent rejection (alpha > 1),
    exponential-mixture rejection (alpha < 1)."""
    if alpha == 1.:
        return -math.log(1. - uniform01(rng)) * beta
    if alpha > 1.:
        while True:
            y = math.tan(PI * uniform01(rng))
            x = math.sqrt(2. * alpha - 1.) * y + alpha - 1.
            if x <= 0.:
                continue
            if uniform01(rng) > (1. + y * y) * math.exp((alpha - 1.) * math.log(x / (alpha - 1.))
                                                          - math.sqrt(2. * alpha - 1.) * y):
                continue
            return x * beta
    p = math.exp(1.) / (alpha + math.exp(1.))
    while True:
        u = uniform01(rng)
        y = -math.log(1. - uniform01(rng))
        if u < p:
            x = math.exp(-y / alpha)
            q = p * math.exp(-x)
        else:
            x = 1. + y
            q = p + (1. - p) * math.pow(x, alpha - 1.)
        if u < q:
            return x * beta


def gaussian_noise(image, rng, sigma):
    """GaussianNoise._applyTo (noise.py:259-263): N(0, sigma) per pixel in row-major order,
    cast to the image dtype and added."""
    g = ONormal(0., sigma)
    noise = np.array([g(rng) for _ in range(image.size)]).reshape(image.shape)
    image += noise.astype(image.dtype)
    return image


def variable_gaussian_noise(image, rng, var):
    """VariableGaussianNoise._applyTo (noise.py:633-636, GaussianDeviate::generateFromVariance,
    Random.cpp:402-450): a fresh unit normal (pair cache cleared) per pixel in row-major order
    times sqrt(variance), cast to the image dtype and added."""
    g = ONormal(0., 1.)
    v = np.asarray(var, dtype=np.float64).reshape(-1)
    noise = np.array([g(rng) * math.sqrt(v[i]) for i in range(image.size)]).reshape(image.shape)
    image += noise.astype(image.dtype)
    return image


def _poisson_fill(noise, rng):
    pd = OPoissonDeviate(rng)
    flat = noise.reshape(-1)
    for i in range(flat.size):
        if flat[i] > 0.:
            pd.set_mean(flat[i])
            flat[i] = pd()


def poisson_noise(image, rng, sky_level=0.):
    """PoissonNoise._applyTo (noise.py:331-356)."""
    noise = image.astype(np.float64)
    # numpy scalar arithmetic as in the reference (a float image gives frac_sky = 0)
    frac_sky = sky_level - image.dtype.type(sky_level)
    int_sky = sky_level - frac_sky
    if sky_level != 0.:
        noise += sky_level
    noise = noise.clip(0.)
    _poisson_fill(noise, rng)
    if frac_sky != 0.:
        noise -= frac_sky
    np.copyto(image, noise, casting='unsafe')
    if int_sky != 0.:
        _isub(image, int_sky)
    return image


def _isub(image, a):
    """Image.__isub__ with a scalar (image.py:1666-1678)."""
    if type(a) == image.dtype.type:
        image[:, :] -= a
    else:
        r = image - a
        if image.dtype.kind in 'iu':
            r = np.around(r)
        image[:, :] = r.astype(image.dtype, copy=False)


def ccd_noise(image, rng, sky_level=0., gain=1., read_noise=0.):
    """CCDNoise._applyTo (noise.py:463-486)."""
    noise = image.astype(np.float64)
    frac_sky = sky_level - image.dtype.type(sky_level)
    int_sky = sky_level - frac_sky
    if sky_level != 0.:
        noise += sky_level
    if gain > 0.:
        noise *= gain
        noise = noise.clip(0.)
        _poisson_fill(noise, rng)
        noise /= gain
    if read_noise > 0.:
        g = ONormal(0., read_noise / gain if gain > 0. else read_noise)
        flat = noise.reshape(-1)
        for i in range(flat.size):
            flat[i] += g(rng)
    if frac_sky != 0.:
        noise -= frac_sky
    np.copyto(image, noise, casting='unsafe')
    if int_sky != 0.:
        _isub(image, int_sky)
    return image
