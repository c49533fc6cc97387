// FP64 on-device construction of the FT tables and the leaf sizing (stepk / maxk).
//
//   ogata_*      Ogata (2005) nodes and weights for h = 2^-5 .. 2^-20, plus the first 10^6
//                zeros of J0, built once per device (gsb_init).
//   hankel_*     the reference's adaptive Hankel transform (src/math/Hankel.cpp:179-249),
//                one warp per transform, terms summed 32 at a time with a warp prefix sum.
//   sersic_*     SersicInfo (src/SBSersic.cpp:301-667): HLR and missing-flux radii by
//                Brent, the ln k table of the Hankel transform, its high-k fit and maxk,
//                and the natural cubic spline (src/Table.cpp:634-686).
//   kolmogorov_* KolmogorovInfo stepk (src/SBKolmogorov.cpp:338-420).
//   prepare_*    per-leaf derived constants and stepk / maxk.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gsb_internal.cuh"
#include "gsb_interp.cuh"

namespace gsb {

namespace {

constexpr int kLevMin = 5;
constexpr int kMaxRounds = 128;      // rounds of ln k nodes per table build (status flags)
// ln k nodes per table and round: a table's nodes past its stopping point are integrated only
// up to the end of the round in which its scan stops (even: the nodes go in pairs)
constexpr int kTableRound = 64;
constexpr int kLevMax = 20;
constexpr long long kNroot = 1000000;

// 2^(j/256), j = 0..255, correctly rounded (computed on the host in extended precision by
// ogata_init): the exponential table of the quadrature kernels' exp_tab256_core.
__device__ double g_exp2_256[256];

// The same method with a 256-entry table 2^(j/256) (`tab`, correctly rounded, filled by the
// caller): |r| <= ln2/512, so the degree-4 Taylor polynomial of e^r suffices (truncation
// < 4e-17 relative), two fused multiply-adds fewer than exp_tab_core.  For the quadrature
// kernels, which evaluate billions of exponentials per table build.
__device__ __forceinline__ double exp_tab256_core(double x, const double* tab)
{
    const double kShift = 6755399441055744.0;               // 1.5 * 2^52
    const double s = __dadd_rn(__dmul_rn(x, 369.3299304675746), kShift);   // 256 / ln2
    const int n = __double2loint(s);
    const double t = s - kShift;
    double r = fma(-t, 0.0027076061740622863, x);            // ln2/256, leading double
    r = fma(-t, 9.058776616587108e-20, r);                   // ln2/256, remainder
    const int j = n & 255;
    const int m = n >> 8;
    double p = fma(r, 1. / 24., 1. / 6.);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.);
    p = fma(p, r, 1.);
    const double v = tab[j] * p;
    return __hiloint2double(__double2hiint(v) + (m << 20), __double2loint(v));
}

__device__ __forceinline__ double exp_tab256_neg(double x, const double* tab)
{
    return exp_tab256_core(fmax(x, -708.), tab);
}

__global__ void ogata_root_kernel(double2* root, long long nroot)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= nroot) return;
    const double z = bessel_j0_zero(i + 1);
    root[i] = make_double2(z, y0(z) / j1(z));
}

// Node i of level h: (log x, w) with x = pi/h psi(h xi) and the Ogata weight w.
__device__ inline double2 ogata_node(const double2* root, double h, long long i)
{
    const double2 r = root[i];
    const double t = h * r.x / kPi;
    const double x = kPi / h * ogata_psi(t);
    const double w = r.y * kPi * x * j0(x) * ogata_dpsi(t);
    return make_double2(log(x), w);
}

__global__ void ogata_level_kernel(double2* xw, const double2* root, double h, long long n)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    xw[i] = ogata_node(root, h, i);
}

__device__ inline double warp_total(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Running-sum estimate refresh: every chunk for the first kEagerChunks chunks (short sums stop
// there), then every kLazyChunks chunks.
constexpr int kEagerChunks = 2;
constexpr int kLazyChunks = 16;

// Sum_i w_i f(x_i / k) / k^2 for h = 2^-lev with the reference's stopping rule: stop at the
// first term whose magnitude is below 1e-15 |running sum| (Hankel.cpp:117-141).  The integrand
// is called with log(x_i / k) = log x_i - log k (nodes store log x), which spares a division
// and a logarithm per term.  Each lane keeps the sum of its own terms; the warp total is formed
// only every few chunks, and the stopping test uses that total.  The stop can therefore move by
// terms below 1e-15 of the sum, which changes the result only at that level.
template <class F>
__device__ double warp_ogata_sum(const OgataTables& og, const F& f, double k, int lev)
{
    const int lane = threadIdx.x & 31;
    const double h = ldexp(1.0, -lev);
    const long long nmax = (long long)fmin(kPi / h, 1e6);
    const bool tab = lev >= og.lev_min && lev <= og.lev_max;
    const double2* xw = tab ? og.xw + og.off[lev - og.lev_min] : nullptr;
    const double logk = log(k);
    double acc = 0., thresh = 0.;
    int chunk = 0;
    for (long long base = 0; base < nmax; base += 32, ++chunk) {
        const long long i = base + lane;
        const bool valid = i < nmax;
        double step = 0.;
        if (valid) {
            const double2 n = tab ? xw[i] : ogata_node(og.root, h, i);
            step = n.y * f(n.x - logk);
        }
        const unsigned mask = __ballot_sync(0xffffffffu, valid && fabs(step) < thresh);
        if (mask) {
            const int last = __ffs(mask) - 1;
            return warp_total(acc + (lane <= last ? step : 0.)) / (k * k);
        }
        acc += step;
        if (chunk < kEagerChunks || (chunk % kLazyChunks) == kLazyChunks - 1)
            thresh = 1e-15 * fabs(warp_total(acc));
    }
    return warp_total(acc) / (k * k);
}

// AdaptiveHankelIntegrator::integrate (Hankel.cpp:179-219).  `status` is set to 1 when
// the halving ran past 2^-60 without meeting the tolerance.
template <class F>
__device__ double warp_hankel(const OgataTables& og, const F& f, double k, double relerr,
                              double abserr, int* status)
{
    int lev = 5;
    double h0 = 1. / 32.;
    while (h0 > 100. * k && lev < 60) { h0 *= 0.5; ++lev; }
    double ans0 = warp_ogata_sum(og, f, k, lev);
    double ans1 = warp_ogata_sum(og, f, k, lev + 1);
    double err = fabs(ans1 - ans0);
    while ((err > relerr * ans1 && (err > abserr || fabs(ans1) > 2. * fabs(ans0))) || ans1 == 0.) {
        ++lev;
        if (lev > 60) { if (status) *status = 1; break; }
        ans0 = ans1;
        ans1 = warp_ogata_sum(og, f, k, lev + 1);
        err = fabs(ans1 - ans0);
    }
    return ans1;
}

// The Sersic integrand exp(-r^(1/n)) is evaluated inline by the node-pair quadrature below, with
// log r = log x_i - log k; its n-derivative along the table's moving grid (GSB_TABLES_DN): the
// quadrature sum T(k) = sum_j w_j f(x_j / k) has dT/dn along k = k(n) with d ln k / dn = c equal
// to sum_j w_j [df/dn - c r df/dr](x_j / k); df/dn = f u ln r / n^2, r df/dr = -f u / n,
// u = r^(1/n).

// Two adjacent ln k nodes of one Sersic table in one warp (k0 < k1 = k0 e^dlogk): the terms
// of both sums at one level share the node load (log x_i, w_i) and the inner exponential,
//   u0 = (x_i / k0)^(1/n) = exp((log x_i - log k0) / n),   u1 = u0 * exp((log k0 - log k1) / n),
// so a pair of terms costs three exponentials instead of four, and each lane carries two
// independent outer exponentials.  Each sum keeps warp_ogata_sum's stopping rule on its own
// running total (the loop runs until both have stopped; a stopped or inactive sum skips its
// outer exponential, a warp-uniform branch).  Node 0's terms are warp_ogata_sum's; node 1's
// u differs from a direct exponential by the rounding of one product (~1e-16 relative), the
// size of the exponential's own rounding.  The inner argument is bounded (|log x_i - log k|
// / n < 100 for the tabulated nodes and the tables' k range), so it takes no range test.
// (Groups of four nodes per warp share more, but their state no longer fits the 64 registers
// that four 256-thread blocks per SM allow, and they measured slower.)
// DN: also the d/dn integrand on the same nodes, f u / n (log r / n + c) with c = dfront/dn (its
// sums stop where the value sums stop, the halving follows the values), returned through dout.
template <bool TAB, bool DN = false>
__device__ __forceinline__ double2 warp_ogata_sum_pair(const OgataTables& og, double invn, double c1,
                                                       double logk0, double logk1, int lev, bool act0,
                                                       bool act1, const double* etab, double dnc = 0.,
                                                       double2* dout = nullptr)
{
    const int lane = threadIdx.x & 31;
    const double h = ldexp(1.0, -lev);
    const int nmax = (int)fmin(kPi / h, 1e6);
    const double2* xw = TAB ? og.xw + og.off[lev - og.lev_min] : nullptr;
    double acc0 = 0., acc1 = 0., th0 = 0., th1 = 0.;
    double dacc0 = 0., dacc1 = 0.;
    int chunk = 0;
    for (int base = 0; base < nmax; base += 32, ++chunk) {
        const int i = base + lane;
        const bool valid = i < nmax;
        double s0 = 0., s1 = 0., ds0 = 0., ds1 = 0.;
        if (valid) {
            const double2 n = TAB ? xw[i] : ogata_node(og.root, h, i);
            const double lr0 = n.x - logk0;
            const double u0 = exp_tab256_core(lr0 * invn, etab);
            if (act0) {
                const double f = exp_tab256_neg(-u0, etab);
                s0 = n.y * f;
                if (DN) ds0 = s0 * u0 * invn * (lr0 * invn + dnc);
            }
            if (act1) {
                const double u1 = u0 * c1;
                const double f = exp_tab256_neg(-u1, etab);
                s1 = n.y * f;
                if (DN) ds1 = s1 * u1 * invn * ((n.x - logk1) * invn + dnc);
            }
        }
        if (act0) {
            const unsigned m0 = __ballot_sync(0xffffffffu, valid && fabs(s0) < th0);
            if (m0) {
                const bool in = lane <= __ffs(m0) - 1;
                acc0 = warp_total(acc0 + (in ? s0 : 0.));
                if (DN) dacc0 = warp_total(dacc0 + (in ? ds0 : 0.));
                act0 = false;
            } else {
                acc0 += s0;
                if (DN) dacc0 += ds0;
            }
        }
        if (act1) {
            const unsigned m1 = __ballot_sync(0xffffffffu, valid && fabs(s1) < th1);
            if (m1) {
                const bool in = lane <= __ffs(m1) - 1;
                acc1 = warp_total(acc1 + (in ? s1 : 0.));
                if (DN) dacc1 = warp_total(dacc1 + (in ? ds1 : 0.));
                act1 = false;
            } else {
                acc1 += s1;
                if (DN) dacc1 += ds1;
            }
        }
        if (!(act0 || act1)) break;
        if (chunk < kEagerChunks || (chunk % kLazyChunks) == kLazyChunks - 1) {
            if (act0) th0 = 1e-15 * fabs(warp_total(acc0));
            if (act1) th1 = 1e-15 * fabs(warp_total(acc1));
        }
    }
    // sums that ran to nmax without stopping
    if (act0) { acc0 = warp_total(acc0); if (DN) dacc0 = warp_total(dacc0); }
    if (act1) { acc1 = warp_total(acc1); if (DN) dacc1 = warp_total(dacc1); }
    const double k0 = exp(logk0), k1 = exp(logk1);
    if (DN) *dout = make_double2(dacc0 / (k0 * k0), dacc1 / (k1 * k1));
    return make_double2(acc0 / (k0 * k0), acc1 / (k1 * k1));
}

// The reference's halving and stopping rule (AdaptiveHankelIntegrator::integrate,
// Hankel.cpp:179-219) for both nodes of the pair, advanced over one common level index L:
// node j starts at its own level s_j (h0 = 1/32 halved while h0 > 100 k_j; s_1 <= s_0 since
// k_1 > k_0), takes the sum at every level from s_j on (ans0 <- ans1, ans1 <- sum(L)) and
// stops at the first level where the reference's test passes; a node that has stopped, or has
// not started, does not contribute to the level's sums.  The running answers live in this
// warp's shared-memory slot `a` (ans0, ans1 of node 0, then of node 1) rather than in
// registers across the term loop.  has1 = false integrates node 0 alone.
template <bool DN = false>
__device__ double2 warp_hankel_pair(const OgataTables& og, double invn, double logk0, double logk1,
                                    bool has1, double relerr, double abserr, int* status, double* a,
                                    const double* etab, double dnc = 0.)
{
    const int lane = threadIdx.x & 31;
    const double k0 = exp(logk0), k1 = exp(logk1);
    int s0 = 5, s1 = 5;
    for (double h0 = 1. / 32.; h0 > 100. * k0 && s0 < 60; h0 *= 0.5) ++s0;
    for (double h0 = 1. / 32.; h0 > 100. * k1 && s1 < 60; h0 *= 0.5) ++s1;
    const double c1 = exp((logk0 - logk1) * invn);
    auto more = [&](double x0, double x1) {
        const double err = fabs(x1 - x0);
        return (err > relerr * x1 && (err > abserr || fabs(x1) > 2. * fabs(x0))) || x1 == 0.;
    };
    bool run0 = true, run1 = has1;
    for (int L = has1 ? min(s0, s1) : s0; run0 || run1; ++L) {
        // the reference halves until its level counter passes 60: the last sum is at 61
        if (L > 61) { if (status) *status = 1; break; }
        const bool g0 = run0 && L >= s0, g1 = run1 && L >= s1;
        double2 d = make_double2(0., 0.);
        const double2 r = (L >= og.lev_min && L <= og.lev_max)
                              ? warp_ogata_sum_pair<true, DN>(og, invn, c1, logk0, logk1, L, g0, g1, etab, dnc, &d)
                              : warp_ogata_sum_pair<false, DN>(og, invn, c1, logk0, logk1, L, g0, g1, etab, dnc, &d);
        __syncwarp();
        if (lane == 0) {
            if (g0) { a[0] = a[1]; a[1] = r.x; if (DN) a[5] = d.x; }
            if (g1) { a[2] = a[3]; a[3] = r.y; if (DN) a[7] = d.y; }
        }
        __syncwarp();
        if (g0 && L > s0) run0 = more(a[0], a[1]);
        if (g1 && L > s1) run1 = more(a[2], a[3]);
    }
    __syncwarp();
    return make_double2(a[1], a[3]);
}

// Truncated Hankel transform (math::hankel_trunc, src/math/Hankel.cpp:249-255) of a radial
// profile f, as SersicInfo::buildFT (src/SBSersic.cpp:453-457) and SBMoffat::setupFT
// (src/SBMoffat.cpp:587-592) call it:
//   I(k) = int_0^t r f(r) J0(k r) dr,   f = exp(-r^(1/n)) (Sersic), (1 + r^2)^-beta (Moffat).
// The reference integrates adaptively (Gauss-Kronrod-Patterson to relerr 1e-6); here the
// integral is taken to near FP64 precision by 16-point Gauss-Legendre on panels between
// consecutive zeros of J0(k r) (the first interval graded toward r = 0 in 48 halvings, where
// the Sersic r^(1/n) has its cusp), so the two agree to the reference's integration error.
// One warp per node: lanes 0-15 and 16-31 take two panels at a time, one Legendre node each.
__device__ inline void gauss_legendre16(int q, double* x, double* w)
{
    // node q of P_16 by Newton's method from the Tricomi estimate, weight 2 / ((1 - x^2) P'^2)
    double z = cos(kPi * (q + 0.75) / 16.5), dp = 1.;
    for (int it = 0; it < 10; ++it) {
        double p0 = 1., p1 = z;
        for (int m = 2; m <= 16; ++m) {
            const double p2 = ((2. * m - 1.) * z * p1 - (m - 1.) * p0) / m;
            p0 = p1;
            p1 = p2;
        }
        dp = 16. * (z * p1 - p0) / (z * z - 1.);
        z -= p1 / dp;
    }
    *x = z;
    *w = 2. / ((1. - z * z) * dp * dp);
}

struct SersicRadial {
    double invn;
    __device__ double operator()(double r) const { return exp(-pow(r, invn)); }
};
struct MoffatRadial {
    double beta;
    __device__ double operator()(double r) const { return pow(1. + r * r, -beta); }
};

template <class F>
__device__ double warp_hankel_trunc(const OgataTables& og, const F& f, double k, double t, int* status)
{
    const int lane = threadIdx.x & 31, half = lane >> 4;
    double xq, wq;
    gauss_legendre16(lane & 15, &xq, &wq);
    const double rfirst = fmin(og.root[0].x / k, t);
    constexpr int M = 48;
    double acc = 0.;
    for (long long jp = 0;; jp += 2) {
        // panel jp (lanes 0-15) and jp + 1 (lanes 16-31)
        const long long j = jp + half;
        double a, b;
        bool live;
        if (j < M) {
            a = ldexp(rfirst, int(j - M));
            b = ldexp(rfirst, int(j + 1 - M));
            live = true;
        } else {
            const long long m = j - M;                      // panel between zeros m and m + 1 (1-based)
            if (m + 1 >= og.nroot) { if (status) *status = 1; live = false; a = b = t; }
            else {
                a = m == 0 ? rfirst : og.root[m - 1].x / k;
                b = fmin(og.root[m].x / k, t);
                live = a < t;
            }
        }
        if (!__any_sync(0xffffffffu, live)) break;
        if (live) {
            const double h = 0.5 * (b - a), r = a + h * (1. + xq);
            acc += wq * h * r * f(r) * j0(k * r);
        }
    }
    return warp_total(acc);
}

struct KolmKValue {
    __device__ double operator()(double logk) const { return exp_tab(-exp_tab(logk * (5. / 3.))); }
};

// (1 - P(2n, z)) Gamma(2n) - target   (SersicMissingFlux, SBSersic.cpp:541-556)
struct SersicMissingFlux {
    double twon, gam, target;
    __device__ double operator()(double z) const { return (1. - gamma_p(twon, z)) * gam - target; }
};

// CalculateB (SBSersic.cpp:627-658)
__device__ RootResult sersic_b(double n, double gamma2n, double flux_fraction)
{
    const double invn = 1. / n, invnsq = invn * invn;
    const double b1 = 2. * n - 1. / 3.;
    const double b2 = b1 + (8. / 405.) * invn + (46. / 25515.) * invnsq +
                      (131. / 1148175.) * invn * invnsq;
    SersicMissingFlux f{2. * n, gamma2n, (1. - 0.5 * flux_fraction) * gamma2n};
    return solve_bracket_lower_limit(f, b1, b2, 0.);
}

// calculateMissingFluxRadius (SBSersic.cpp:558-625); result in units of r0.
__device__ RootResult sersic_missing_flux_radius(double n, double gamma2n, double b,
                                                 double missing_frac)
{
    const double missing_flux = missing_frac * gamma2n;
    double z1 = -log(missing_flux);
    double z;
    if (n == 0.5) {
        z = z1;
    } else {
        z = 4. * (n + 1.);
        const double twonm1 = 2. * n - 1.;
        double z2 = z1 + twonm1 * log(z) + twonm1 / z + twonm1 * (2. * n - 3.) / (2. * z * z);
        if (z2 > z1 && z2 - z1 < 0.01) z2 = z1 + 0.01;
        else if (z2 < z1 && z2 - z1 > -0.01) z2 = z1 - 0.01;
        if (z1 < 0.) z1 = b;
        SersicMissingFlux f{2. * n, gamma2n, missing_flux};
        RootResult r = solve_bracket_upper(f, z1, z2);
        if (!r.ok) return {0., false};
        z = r.x;
    }
    return {pow(z, n), true};
}

// Truncated Sersic sizes (sersic.py:218-247 with SersicTruncatedScale / SersicIntegratedFlux,
// src/SBSersic.cpp:332-336, 688-775): per profile (n, size, trunc, flags) with flags bit 0 = size
// is a half-light radius, bit 1 = flux_untruncated:
//   r0 = size                                 (scale radius given)
//   r0 = hlr / b_untruncated(n)^n             (hlr given, flux_untruncated)
//   r0 = hlr * CalculateTruncatedScale(n, b, trunc / hlr)   (hlr of the truncated profile)
// and the flux fraction gamma_p(2n, (trunc / r0)^(1/n)) inside trunc.
struct SersicTruncatedHLR {
    double twon, x, gam;
    __device__ double operator()(double b) const
    { return (2. * gamma_p(twon, b) - gamma_p(twon, x * b)) * gam; }
};

__global__ void sersic_truncation_kernel(const double* in, int count, double* out, int* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double n = in[4 * i], size = in[4 * i + 1], trunc = in[4 * i + 2];
    const int flags = int(in[4 * i + 3]);
    const double gamma2n = tgamma(2. * n);
    double r0 = size;
    if (flags & 1) {
        const RootResult rb = sersic_b(n, gamma2n, 1.);
        if (!rb.ok) { atomicOr(status, 1); return; }
        if (flags & 2) {
            r0 = size / pow(rb.x, n);
        } else {
            // b solves gamma_p(2n, b) = gamma_p(2n, x b) / 2, x = (trunc / hlr)^(1/n), bracketed
            // by the asymptotic guess (or b / 2) and the untruncated b (SBSersic.cpp:688-768)
            const double x = pow(trunc / size, 1. / n);
            double b1 = (log(0.5) + (2. * n - 1.) * log(x)) / (x - 1.);
            if (b1 < 1e-3 * rb.x) b1 = 0.5 * rb.x;
            const RootResult rt = solve_bracket_lower_limit(SersicTruncatedHLR{2. * n, x, gamma2n}, b1, rb.x, 0.);
            if (!rt.ok) { atomicOr(status, 1); return; }
            r0 = size / pow(rt.x, n);
        }
    }
    out[2 * i] = r0;
    out[2 * i + 1] = gamma_p(2. * n, pow(trunc / r0, 1. / n));
}

__global__ void sersic_setup_kernel(const double* n_arr, const double* trunc_arr, int count, gsb_gsparams gsp,
                                    double* header, int stride, double* dheader)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    double* H = header + (size_t)s * kSersicHeader;
    const double n = n_arr[s];
    const double trunc = trunc_arr ? trunc_arr[s] : 0.;      // in units of r0
    const double gamma2n = tgamma(2. * n);
    double gamma4n = tgamma(4. * n);
    double gamma6n = tgamma(6. * n);
    double gamma8n = tgamma(8. * n);
    // truncated profiles (SBSersic.cpp:332-352, 393-424): the flux fraction inside trunc and the
    // moments of the truncated profile
    double ff = 1.;
    if (trunc > 0.) {
        const double z = pow(trunc, 1. / n);
        ff = gamma_p(2. * n, z);
        gamma4n *= gamma_p(4. * n, z);
        gamma6n *= gamma_p(6. * n, z);
        gamma8n *= gamma_p(8. * n, z);
    }
    // buildFT low-k series (SBSersic.cpp:386-424)
    const double kderiv2 = -gamma4n / (4. * gamma2n) / ff;
    const double kderiv4 = gamma6n / (64. * gamma2n) / ff;
    const double kderiv6 = gamma8n / (2304. * gamma2n) / ff;
    const double kmin = pow(gsp.kvalue_accuracy / kderiv6, 1. / 6.);
    const double dlogk = gsp.table_spacing * sqrt(sqrt(gsp.kvalue_accuracy / 10.));
    int ncand = 0;
    const double logk_end = log(500.);
    for (double logk = log(kmin) - 0.001; logk < logk_end && ncand < stride; logk += dlogk)
        ++ncand;
    int status = 0;
    RootResult rb = sersic_b(n, gamma2n, ff);
    if (!rb.ok) status = 2;
    const double b = rb.x;
    // stepK (SBSersic.cpp:304-318): the untruncated missing-flux radius (its lower bracket falls
    // back to the profile's own b, :589-592), capped at trunc
    RootResult rr = sersic_missing_flux_radius(n, gamma2n, b, gsp.folding_threshold);
    if (!rr.ok) status = 3;
    double R = rr.x;
    if (trunc > 0. && trunc < R) R = trunc;
    R = fmax(R, gsp.stepk_minimum_hlr);
    H[kSH_N] = n;
    H[kSH_NUSED] = 0;
    H[kSH_FRONT] = log(kmin) - 0.001;
    H[kSH_DA] = dlogk;
    H[kSH_KSQMIN] = kmin * kmin;
    H[kSH_KSQMAX] = 0.;
    H[kSH_KD2] = kderiv2;
    H[kSH_KD4] = kderiv4;
    H[kSH_HIGHA] = 0.;
    H[kSH_HIGHB] = 0.;
    H[kSH_MAXK] = kmin;
    H[kSH_STEPK] = kPi / R;
    H[kSH_RE] = pow(b, n);
    H[kSH_DLOGK] = dlogk;
    H[kSH_NCAND] = ncand;
    H[kSH_STATUS] = status;
    H[kSH_TRUNC] = trunc;
    H[kSH_FLUXFRAC] = ff;
    if (dheader) {
        // d/dn of the low-k coefficients (ratios of Gamma functions) and of ln(r_e / r0) =
        // n ln b, with db/dn from P(2n, b) = 1/2 by implicit differentiation.
        double* D = dheader + (size_t)s * kSersicDHeader;
        const double psi2 = digamma(2. * n);
        D[kSD_DKD2] = kderiv2 * (4. * digamma(4. * n) - 2. * psi2);
        D[kSD_DKD4] = kderiv4 * (6. * digamma(6. * n) - 2. * psi2);
        D[kSD_DHIGHA] = 0.;
        D[kSD_DHIGHB] = 0.;
        // front = ln k_min - 0.001 with k_min = (kvalue_accuracy / kderiv6)^(1/6)
        D[kSD_DFRONT] = -(8. * digamma(8. * n) - 2. * psi2) / 6.;
        const double dPdb = exp(-b + (2. * n - 1.) * log(b) - lgamma(2. * n));
        const double dbdn = -2. * gamma_p_da(2. * n, b) / dPdb;
        D[kSD_DLNRE] = log(b) + n * dbdn / b;
    }
}

// Running state of the serial part of buildFT for one table (SBSersic.cpp:436-509): the
// maxk bookkeeping and the 10-point high-k least-squares fit, advanced one round of nodes at a
// time so that nodes past the stopping point are never integrated.
struct SersicScan {
    double sf, skf, sk, sk2, maxk, ksq_max, a, b;
    double fit[10];
    int fit_size, fit_head, n_correct, found, nused, done;
};

__global__ void sersic_scan_init_kernel(const double* header, int count, SersicScan* scan)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    SersicScan& S = scan[s];
    S.sf = S.skf = S.sk = S.sk2 = 0.;
    S.maxk = sqrt(header[(size_t)s * kSersicHeader + kSH_KSQMIN]);
    S.ksq_max = -1.;
    S.a = S.b = 0.;
    S.fit_size = S.fit_head = S.n_correct = S.found = S.nused = 0;
    S.done = int(header[(size_t)s * kSersicHeader + kSH_NCAND]) < 2 ? 1 : 0;
}

// One warp per node of this round for the truncated tables (trunc > 0; the pair kernel skips
// them): the truncated Hankel transform / hankel_norm, hankel_norm = flux fraction n Gamma(2n).
__global__ void __launch_bounds__(256) sersic_trunc_nodes_kernel(const double* header, int count, int i0,
                                    int nround, const __grid_constant__ OgataTables og, const SersicScan* scan,
                                    double* vals, int stride, const int* prev_live, int* status_out)
{
    if (prev_live && *prev_live == 0) return;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long s = warp / nround;
    const int i = i0 + int(warp % nround);
    if (s >= count) return;
    const double* H = header + s * kSersicHeader;
    if (H[kSH_TRUNC] <= 0. || scan[s].done) return;
    if (i >= int(H[kSH_NCAND])) return;
    const double n = H[kSH_N];
    const double k = exp(H[kSH_FRONT] + i * H[kSH_DLOGK]);
    const double hankel_norm = H[kSH_FLUXFRAC] * n * tgamma(2. * n);
    int st = 0;
    const double v = warp_hankel_trunc(og, SersicRadial{1. / n}, k, H[kSH_TRUNC], &st) / hankel_norm;
    if ((threadIdx.x & 31) == 0) {
        vals[s * stride + i] = v;
        if (st) atomicOr(status_out, 1);
    }
}

// One warp per pair of adjacent nodes (i, i + 1) of this round: Hankel transform / hankel_norm at
// k_i, k_{i+1} through warp_hankel_pair; DN: with the d/dn values of the same nodes.
// prev_live (the previous round's scan flag) is zero once every table has stopped: the launch
// then returns at once.
template <bool DN>
__global__ void __launch_bounds__(256, 4) sersic_nodes_pair_kernel(const double* header, int count, int i0,
                                    int nround, gsb_gsparams gsp, const __grid_constant__ OgataTables og,
                                    const SersicScan* scan, double* vals, int stride,
                                    const int* prev_live, int* status_out, const double* dheader,
                                    double* dvals)
{
    if (prev_live && *prev_live == 0) return;
    // the exponential's 2^(j/256) table, read three times per pair of terms, from shared memory
    __shared__ double etab[256];
    etab[threadIdx.x] = g_exp2_256[threadIdx.x];
    __syncthreads();
    const int npair = (nround + 1) / 2;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    // slots hold ascending n; the costly large-n tables are taken first so that they do not
    // form the tail of the launch
    const long long s = count - 1 - warp / npair;
    const int i = i0 + 2 * int(warp % npair);
    if (s < 0) return;
    if (scan[s].done) return;
    const double* H = header + s * kSersicHeader;
    if (H[kSH_TRUNC] > 0.) return;          // sersic_trunc_nodes_kernel
    const int ncand = int(H[kSH_NCAND]);
    if (i >= ncand) return;
    const bool has1 = i + 1 < ncand && i + 1 < i0 + nround;
    const double n = H[kSH_N];
    const double logk0 = H[kSH_FRONT] + i * H[kSH_DLOGK];
    const double logk1 = H[kSH_FRONT] + (i + 1) * H[kSH_DLOGK];
    const double hankel_norm = n * tgamma(2. * n);
    __shared__ double ans[8][DN ? 8 : 4];  // the running answers of each warp's pair
    double* a = ans[(threadIdx.x >> 5) & 7];
    int st = 0;
    const double dnc = DN ? dheader[s * kSersicDHeader + kSD_DFRONT] : 0.;
    const double2 v = warp_hankel_pair<DN>(og, 1. / n, logk0, logk1, has1, gsp.integration_relerr,
                                           gsp.integration_abserr * hankel_norm, &st, a, etab, dnc);
    if ((threadIdx.x & 31) == 0) {
        const double v0 = v.x / hankel_norm, v1 = v.y / hankel_norm;
        vals[s * stride + i] = v0;
        if (has1) vals[s * stride + i + 1] = v1;
        if (DN) {
            // node value y = v k^2 = T(k) / norm with norm = n Gamma(2n) and k = k_i(n):
            // dy/dn = (dT/dn) / norm - y (1/n + 2 psi(2n)), dT/dn from the second integrand.
            const double q = 1. / n + 2. * digamma(2. * n);
            const double k0 = exp(logk0), k1 = exp(logk1);
            dvals[s * stride + i] = (a[5] / hankel_norm - v0 * q) * k0 * k0;
            if (has1) dvals[s * stride + i + 1] = (a[7] / hankel_norm - v1 * q) * k1 * k1;
        }
        if (st) atomicOr(status_out, 1);
    }
}

// live_out is set when a table still needs nodes after this round; a zero prev_live (the
// previous round's flag) means every table has stopped and the launch returns at once.
__global__ void sersic_scan_kernel(const double* header, int count, int stride, int i0, int nround,
                                   gsb_gsparams gsp, const double* vals, double4* nodes,
                                   SersicScan* scan, const double* dvals, double4* dnodes,
                                   const int* prev_live, int* live_out)
{
    if (prev_live && *prev_live == 0) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    if (scan[s].done) return;
    // the state is advanced in a local copy (the node stores below may alias it as far as the
    // compiler knows, which would send every field access to global memory) and written back
    SersicScan S = scan[s];
    const double* H = header + (size_t)s * kSersicHeader;
    const double* v = vals + (size_t)s * stride;
    double4* nd = nodes + (size_t)s * stride;
    const int ncand = int(H[kSH_NCAND]);
    const double front = H[kSH_FRONT], dlogk = H[kSH_DLOGK];
    const int n_fit = 10;
    const int iend = min(i0 + nround, ncand);
    for (int i = i0; i < iend; ++i) {
        const double logk = front + i * dlogk;
        const double k = exp(logk), ksq = k * k;
        const double val = v[i];
        const double f0 = val * ksq;
        nd[i] = make_double4(logk, f0, 0., 0.);
        if (dnodes) dnodes[(size_t)s * stride + i] = make_double4(logk, dvals[(size_t)s * stride + i], 0., 0.);
        S.nused = i + 1;
        if (fabs(val) > gsp.maxk_threshold) { S.maxk = k; S.n_correct = 0; }
        else {
            S.found = 1;
            const double den = n_fit * S.sk2 - S.sk * S.sk;
            S.a = (S.sf * S.sk2 - S.sk * S.skf) / den;
            S.b = (n_fit * S.skf - S.sk * S.sf) / den;
            const double f0_pred = S.a + S.b / k;
            if (fabs(f0 - f0_pred) / ksq < gsp.kvalue_accuracy) ++S.n_correct;
            else S.n_correct = 0;
            if (S.n_correct >= 5) { S.ksq_max = ksq; S.done = 1; scan[s] = S; return; }
        }
        const double inv_k = 1. / k;
        if (S.fit_size == n_fit) {
            const double k_back = exp(logk - n_fit * dlogk);
            const double f_back = S.fit[S.fit_head];
            const double inv_k_back = 1. / k_back;
            S.sf += f0 - f_back;
            S.skf += f0 * inv_k - f_back * inv_k_back;
            S.sk += inv_k - inv_k_back;
            S.sk2 += inv_k * inv_k - inv_k_back * inv_k_back;
            S.fit[S.fit_head] = f0;
            S.fit_head = (S.fit_head + 1) % n_fit;
        } else {
            S.sf += f0;
            S.skf += f0 * inv_k;
            S.sk += inv_k;
            S.sk2 += inv_k * inv_k;
            S.fit[S.fit_size++] = f0;
        }
    }
    if (iend >= ncand) S.done = 1;
    scan[s] = S;
    if (!S.done && live_out) *live_out = 1;
}

// End of buildFT (SBSersic.cpp:510-537) and the natural spline (Table.cpp:634-686).
// Natural cubic spline second derivatives z of nodes (x, y) (Thomas algorithm; c is scratch).
// TSpline setup, src/Table.cpp:634-686.
__device__ void natural_spline(const double* x, const double* y, double* z, double* c, int N)
{
    for (int i = 0; i < N; ++i) z[i] = 0.;
    if (N == 3) {
        z[1] = 3. * ((y[2] - y[1]) / (x[2] - x[1]) - (y[1] - y[0]) / (x[1] - x[0])) / (x[2] - x[0]);
    } else if (N > 3) {
        for (int i = 1; i <= N - 2; ++i)
            z[i] = 6. * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]));
        double bb = 2. * (x[2] - x[0]);
        for (int i = 1; i <= N - 2; ++i) {
            z[i] /= bb;
            if (i == N - 2) break;
            const double aa = x[i + 1] - x[i];
            const double cc = aa / bb;
            c[i - 1] = cc;
            bb = 2. * (x[i + 2] - x[i]);
            bb -= aa * cc;
            z[i + 1] -= aa * z[i];
        }
        for (int i = N - 3; i > 0; --i) z[i] -= c[i - 1] * z[i + 1];
    }
}

// End of buildFT (SBSersic.cpp:510-537) and the natural spline, one warp per table: the warp
// stages the table's nodes in shared memory (coalesced), lane 0 runs the serial parts there.
// Dynamic shared memory: 4 * stride doubles.
__global__ void __launch_bounds__(32) sersic_finalize_kernel(double* header, int count, int stride,
                                                             gsb_gsparams gsp, const SersicScan* scan,
                                                             double4* nodes, double4* dnodes, double* dheader)
{
    extern __shared__ double fsm[];
    const int s = blockIdx.x;
    const int lane = threadIdx.x;
    if (s >= count) return;
    double* xs = fsm;
    double* ys = xs + stride;
    double* zs = ys + stride;
    double* cs = zs + stride;
    double* H = header + (size_t)s * kSersicHeader;
    double4* nd = nodes + (size_t)s * stride;
    const SersicScan& S = scan[s];
    const int N = S.nused;
    if (N < 2) {
        if (lane == 0) { H[kSH_STATUS] = 5; H[kSH_NUSED] = 0; }
        return;
    }
    const double front = H[kSH_FRONT], dlogk = H[kSH_DLOGK];
    const int n_fit = 10;
    for (int i = lane; i < N; i += 32) {
        const double4 v = nd[i];
        xs[i] = v.x;
        ys[i] = v.y;
    }
    __syncwarp();
    double ksq_max = 0., maxk = 0., a = 0., b = 0.;
    if (lane == 0) {
        ksq_max = S.ksq_max;
        maxk = S.maxk;
        a = S.a;
        b = S.b;
        if (ksq_max <= 0.) ksq_max = exp(2. * xs[N - 1]);
        if (S.found) {
            maxk *= exp(dlogk);
        } else {
            const double den = n_fit * S.sk2 - S.sk * S.sk;
            a = (S.sf * S.sk2 - S.sk * S.skf) / den;
            b = (n_fit * S.skf - S.sk * S.sf) / den;
            maxk = sqrt(a / gsp.maxk_threshold);
            for (int it = 0; it < 3; ++it) maxk = sqrt((a - b / maxk) / gsp.maxk_threshold);
        }
        natural_spline(xs, ys, zs, cs, N);
    }
    __syncwarp();
    // .w: k^2 at the node, for the evaluators' spline offset 0.5 ln(k_i^2 / k^2)
    for (int i = lane; i < N; i += 32) nd[i] = make_double4(xs[i] - front, ys[i], zs[i], exp(2. * xs[i]));
    const double back = xs[N - 1];
    if (dnodes) {
        // The spline is linear in its node values, so d/dn of the interpolant is the spline of
        // the node derivatives on the same grid.  Likewise the high-k fit is linear in the f0
        // values of its window: the 10 nodes before the stopping node, or the last 10 nodes
        // when the scan ran to the end of the candidate grid.
        double4* dn = dnodes + (size_t)s * stride;
        __syncwarp();
        for (int i = lane; i < N; i += 32) cs[i] = ys[i];     // keep f0 for the fit window
        __syncwarp();
        for (int i = lane; i < N; i += 32) ys[i] = dn[i].y;
        __syncwarp();
        double* f0s = zs;   // reuse: z of the main table is already written out
        if (lane == 0) {
            // The fit's 1/k_i move too: d(1/k_i)/dn = -c / k_i with c = dfront/dn.
            double* D = dheader + (size_t)s * kSersicDHeader;
            const double c = D[kSD_DFRONT];
            const int wend = S.ksq_max > 0. ? N - 1 : N;
            const int wbeg = wend - n_fit > 0 ? wend - n_fit : 0;
            double sk = 0., sk2 = 0., sf = 0., skf = 0., dsf = 0., dskf = 0.;
            for (int i = wbeg; i < wend; ++i) {
                const double inv_k = exp(-(front + i * dlogk));
                const double f0 = cs[i], df0 = ys[i];
                sk += inv_k;
                sk2 += inv_k * inv_k;
                sf += f0;
                skf += f0 * inv_k;
                dsf += df0;
                dskf += (df0 - c * f0) * inv_k;
            }
            const double dsk = -c * sk, dsk2 = -2. * c * sk2;
            const double den = n_fit * sk2 - sk * sk, dden = n_fit * dsk2 - 2. * sk * dsk;
            const double na = sf * sk2 - sk * skf, dna = dsf * sk2 + sf * dsk2 - dsk * skf - sk * dskf;
            const double nb = n_fit * skf - sk * sf, dnb = n_fit * dskf - dsk * sf - sk * dsf;
            D[kSD_DHIGHA] = (dna * den - na * dden) / (den * den);
            D[kSD_DHIGHB] = (dnb * den - nb * dden) / (den * den);
            natural_spline(xs, ys, f0s, cs, N);
        }
        __syncwarp();
        for (int i = lane; i < N; i += 32) dn[i] = make_double4(xs[i] - front, ys[i], f0s[i], 0.);
    }
    if (lane != 0) return;
    H[kSH_NUSED] = N;
    H[kSH_DA] = (back - front) / (N - 1);
    H[kSH_KSQMAX] = ksq_max;
    H[kSH_HIGHA] = a;
    H[kSH_HIGHB] = b;
    H[kSH_MAXK] = maxk;
}

// Truncated Moffat FT tables (SBMoffat::setupFT, src/SBMoffat.cpp:565-625).  Per slot
// (beta, t = trunc / rD): the values
//     v(k) = 2 (beta - 1) / F  int_0^t r (1 + r^2)^-beta J0(k r) dr,  F = 1 - (1 + t^2)^(1 - beta)
// on the reference's grid k = 0, dk, 2 dk, ... (its running sum, k < 50), one warp per node for
// all candidate nodes at once; then, per slot, the reference's stopping rule (5 nodes in a row
// with |v| <= kvalue_accuracy end the table), maxk (the last node with |v| > maxk_threshold,
// refined linearly toward the next node) and the natural cubic spline in k^2.
__global__ void moffat_setup_kernel(int count, double* header)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    double* H = header + (size_t)s * kMoffatHeader;
    H[kMH_FLUXFACTOR] = 1. - pow(1. + H[kMH_TRUNC] * H[kMH_TRUNC], 1. - H[kMH_BETA]);
}

__global__ void __launch_bounds__(256) moffat_nodes_kernel(const double* header, int count, const double* kgrid,
                                                           int ncand, const __grid_constant__ OgataTables og,
                                                           double* vals, int* status_out)
{
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long s = warp / ncand;
    const int i = int(warp % ncand);
    if (s >= count) return;
    const double* H = header + s * kMoffatHeader;
    const double b = H[kMH_BETA];
    const double prefactor = 2. * (b - 1.) / H[kMH_FLUXFACTOR];
    int st = 0;
    const double v = prefactor * warp_hankel_trunc(og, MoffatRadial{b}, kgrid[i], H[kMH_TRUNC], &st);
    if ((threadIdx.x & 31) == 0) {
        vals[s * ncand + i] = v;
        if (st) atomicOr(status_out, 1);
    }
}

// One warp per slot; dynamic shared memory 4 * ncand doubles.
__global__ void __launch_bounds__(32) moffat_finalize_kernel(double* header, int count, const double* kgrid,
                                                             int ncand, gsb_gsparams gsp, const double* vals,
                                                             double4* nodes)
{
    extern __shared__ double msm[];
    const int s = blockIdx.x;
    const int lane = threadIdx.x;
    if (s >= count) return;
    double* xs = msm;
    double* ys = xs + ncand;
    double* zs = ys + ncand;
    double* cs = zs + ncand;
    const double* v = vals + (size_t)s * ncand;
    for (int i = lane; i < ncand; i += 32) {
        xs[i] = kgrid[i] * kgrid[i];
        ys[i] = v[i];
    }
    __syncwarp();
    __shared__ int n_used;
    if (lane == 0) {
        double* H = header + (size_t)s * kMoffatHeader;
        // the reference's loop over k: maxk bookkeeping and the stopping rule
        int im = 0, nbelow = 0, N = ncand;
        for (int i = 0; i < ncand; ++i) {
            const double a = fabs(ys[i]);
            if (a > gsp.maxk_threshold) im = i;
            nbelow = a > gsp.kvalue_accuracy ? 0 : nbelow + 1;
            if (nbelow == 5) { N = i + 1; break; }
        }
        double maxk = kgrid[im];
        // the refinement between k1 = maxk and k2 = maxk + dk (both tabulated nodes when k2 < 50,
        // where the spline returns the node values)
        const double k2 = maxk + H[kMH_DK];
        if (k2 < 50. && im + 1 < N) {
            const double f1 = fabs(ys[im]), f2 = fabs(ys[im + 1]);
            maxk = (maxk * (f2 - gsp.maxk_threshold) + k2 * (gsp.maxk_threshold - f1)) / (f2 - f1);
        }
        if (N >= 2) natural_spline(xs, ys, zs, cs, N);
        H[kMH_NUSED] = N;
        H[kMH_KSQMAX] = xs[N - 1];
        H[kMH_MAXK] = maxk;
        if (N < 2) H[kMH_STATUS] = 5;
        n_used = N;
    }
    __syncwarp();
    const int N = n_used;
    double4* nd = nodes + (size_t)s * ncand;
    for (int i = lane; i < N; i += 32) nd[i] = make_double4(xs[i], ys[i], zs[i], 0.);
}

// Scale radius of truncated Moffat profiles from the half-light radius
// (MoffatCalculateScaleRadiusFromHLR, src/SBMoffat.cpp:103-160): Brent on
//     2 f(re) - f(rm) = 0,   f(R) = 1 - (1 + R^2 / rd^2)^(1 - beta),
// bracketed upward from the untruncated radius r1 and 2 r1.
struct MoffatScaleRadiusFunc {
    double re, rm, beta;
    __device__ double operator()(double rd) const
    {
        const double fre = 1. - pow(1. + (re * re) / (rd * rd), 1. - beta);
        const double frm = 1. - pow(1. + (rm * rm) / (rd * rd), 1. - beta);
        return 2. * fre - frm;
    }
};

__global__ void moffat_scale_radius_kernel(const double* in, int count, double* out, int* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double beta = in[3 * i], re = in[3 * i + 1], rm = in[3 * i + 2];
    const double r1 = re / sqrt(pow(0.5, 1. / (1. - beta)) - 1.);
    // beta <= 1 has no finite untruncated radius to start from: the reference's bracketing
    // fails there too
    if (!(r1 > 0.) || !isfinite(r1)) { atomicOr(status, 1); out[i] = 0.; return; }
    if (rm == 0.) { out[i] = r1; return; }
    const RootResult r = solve_bracket_upper(MoffatScaleRadiusFunc{re, rm, beta}, r1, 2. * r1);
    if (!r.ok) { atomicOr(status, 1); out[i] = 0.; return; }
    out[i] = r.x;
}

// KolmogorovInfo: x-space radial profile by Hankel transform of exp(-k^{5/3}) at
// r = exp(-3 + i dlogr); only the last tabulated point matters for stepk.
__global__ void kolmogorov_nodes_kernel(int ncand, double dlogr, gsb_gsparams gsp, const __grid_constant__ OgataTables og,
                                        double* vals, int* status_out)
{
    const int i = int((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    if (i >= ncand) return;
    const double r = exp(-3. + i * dlogr);
    KolmKValue f;
    int st = 0;
    const double v = warp_hankel(og, f, r, gsp.integration_relerr, gsp.integration_abserr, &st) /
                     (2. * kPi);
    if ((threadIdx.x & 31) == 0) {
        vals[i] = v;
        if (st) atomicOr(status_out, 1);
    }
}

__global__ void kolmogorov_finalize_kernel(int ncand, double dlogr, gsb_gsparams gsp,
                                           const double* vals, double* out, double4* nodes, double* scratch)
{
    // the reference's loop: entries (r, f(r)) from r = e^-3 until f r^2 / 1.67 < thresh (that
    // entry included), after the analytic f(0) = XVAL_ZERO (SBKolmogorov.cpp:352-384)
    const double thresh = gsp.shoot_accuracy / (2. * kPi);
    double r1 = 0., F1 = 0.;
    int nused = 0;
    for (int i = 0; i < ncand; ++i) {
        const double r = exp(-3. + i * dlogr);
        r1 = r; F1 = vals[i];
        nused = i + 1;
        if (vals[i] * r * r / 1.67 < thresh) break;
    }
    const double n = 11. / 3.;
    double R = pow(2. * kPi * F1 * pow(r1, n) / ((n - 2.) * gsp.folding_threshold), 1. / (n - 2.));
    const double hlr = 2.992939911888651 * 0.5548101137;
    R = fmax(R, gsp.stepk_minimum_hlr * hlr);
    out[0] = kPi / R;
    // the radial table's natural spline in r (Table::spline, src/Table.cpp:634-686), for the
    // real-space drawing of Kolmogorov leaves
    const int N = nused + 1;
    double* xs = scratch;
    double* ys = xs + N;
    double* zs = ys + N;
    double* cs = zs + N;
    xs[0] = 0.;
    ys[0] = 0.0876786563672346;     // XVAL_ZERO = (3/5) Gamma(6/5) / (2 pi)
    for (int i = 0; i < nused; ++i) { xs[i + 1] = exp(-3. + i * dlogr); ys[i + 1] = vals[i]; }
    natural_spline(xs, ys, zs, cs, N);
    for (int i = 0; i < N; ++i) nodes[i] = make_double4(xs[i], ys[i], zs[i], 0.);
    out[1] = N;
}

// kV2 for the Moffat maxk solve (MoffatMaxKSolver, SBMoffat.cpp:481-520), normalised to 1
// at k = 0, as a function of ksq.
struct MoffatKV2 {
    int mode;
    double nu, thresh;
    __device__ double operator()(double ksq) const
    {
        const double k = sqrt(ksq);
        double v;
        if (mode == 1) v = exp(-k);
        else if (mode == 2) v = exp(-k) * (1. + k);
        else if (mode == 3) v = exp(-k) * (3. + (3. + k) * k) / 3.;
        else v = moffat_kv_fp64(nu, k);
        return v - thresh;
    }
};

struct MoffatRefs {
    const double* header;
    const double4* node;
    int count, stride;
};

struct ImageRefs {
    const ImageSlot* slots;
    const double* info;
    const double2* k64;
    const float2* k32;
    int count;
};

__global__ void prepare_leaves_kernel(const __grid_constant__ gsb_template tpl, int n_stamps, gsb_gsparams gsp,
                                      gsb_leaf* leaves, const double* sersic_header, MoffatRefs moffat,
                                      double kolm_stepk, ImageRefs images, double* info, int* status_out)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)n_stamps * tpl.n_leaves) return;
    const int l = int(idx % tpl.n_leaves);
    gsb_leaf& L = leaves[idx];
    const int type = tpl.leaf_type[l];
    double stepk = 0., maxk = 0.;
    for (int i = 0; i < 8; ++i) L.d[i] = 0.;
    switch (type) {
      case GSB_GAUSSIAN: {
        // gaussian.py:148-155 and SBGaussian.cpp:63-73
        const double sigma = L.p[0];
        L.d[0] = sigma;
        L.d[1] = -2. * log(gsp.kvalue_accuracy);
        L.d[2] = pow(gsp.kvalue_accuracy * 48., 1. / 3.);
        maxk = sqrt(-2. * log(gsp.maxk_threshold)) / sigma;
        const double R = fmax(sqrt(-2. * log(gsp.folding_threshold)),
                              gsp.stepk_minimum_hlr * 1.1774100225154747);
        stepk = kPi / (R * sigma);
        break;
      }
      case GSB_EXPONENTIAL: {
        // exponential.py:131-136, SBExponential.cpp:65-79 and ExponentialInfo :513-543
        const double r0 = L.p[0];
        const double ksq_max = pow(gsp.kvalue_accuracy, -1. / 1.5) - 1.;
        L.d[0] = r0;
        L.d[1] = ksq_max;
        L.d[2] = sqrt(ksq_max);
        maxk = pow(gsp.maxk_threshold, -1. / 3.) / r0;
        const double logx = log(gsp.folding_threshold);
        double R = -logx;
        for (int i = 0; i < 3; ++i) R = log(1. + R) - logx;
        R = fmax(R, gsp.stepk_minimum_hlr * 1.6783469900166605);
        stepk = kPi / R / r0;
        break;
      }
      case GSB_SERSIC: {
        // SBSersic.cpp:71-90 (r0 from hlr via SersicHLR, sersic.py:224-227), :301-324
        const double* H = sersic_header + (size_t)L.table * kSersicHeader;
        const double r0 = (L.flags & GSB_LEAF_SIZE_IS_HLR) ? L.p[1] / H[kSH_RE] : L.p[1];
        L.d[0] = r0;
        maxk = H[kSH_MAXK] / r0;
        stepk = H[kSH_STEPK] / r0;
        if (H[kSH_STATUS] != 0.) atomicOr(status_out, 2);
        break;
      }
      case GSB_MOFFAT: {
        // SBMoffat.cpp:163-244 (kV selection), :481-549 (maxK, stepK)
        const double beta = L.p[0], rD = L.p[1], trunc = L.p[2];
        double maxRrD, flux_factor = 1.;
        L.d[0] = rD;
        L.d[1] = L.flux;
        if (trunc > 0.) {
            // the FT from the slot's spline in k^2 (kV_trunc, SBMoffat.cpp:339-345); the slot
            // must have been built for this (beta, trunc / rD)
            const int slot = L.table;
            if (slot < 0 || slot >= moffat.count) { atomicOr(status_out, 64); break; }
            const double* H = moffat.header + (size_t)slot * kMoffatHeader;
            if (fabs(H[kMH_BETA] - beta) > 1e-12 * fabs(beta) ||
                fabs(H[kMH_TRUNC] - trunc / rD) > 1e-12 * (trunc / rD)) { atomicOr(status_out, 128); break; }
            if (H[kMH_STATUS] != 0.) atomicOr(status_out, 256);
            maxRrD = trunc / rD;
            flux_factor = H[kMH_FLUXFACTOR];
            L.d[2] = 4;
            L.d[3] = H[kMH_DK];
            L.d[4] = H[kMH_KSQMAX];
            L.d[5] = H[kMH_NUSED];
            L.d[6] = __longlong_as_double((long long)(moffat.node + (size_t)slot * moffat.stride));
            maxk = H[kMH_MAXK] / rD;
        } else {
            const double kacc = gsp.kvalue_accuracy;
            int mode = 0;
            double nu = beta - 1.;
            if (fabs(beta - 1.5) < kacc) { mode = 1; }
            else if (fabs(beta - 2.) < kacc) { nu = 1.; }
            else if (fabs(beta - 2.5) < kacc) { mode = 2; }
            else if (fabs(beta - 3.) < kacc) { nu = 2.; }
            else if (fabs(beta - 3.5) < kacc) { mode = 3; }
            else if (fabs(beta - 4.) < kacc) { nu = 3.; }
            L.d[2] = mode;
            L.d[3] = nu;
            L.d[4] = (1. - nu) * log(2.) - lgamma(nu);
            MoffatKV2 f{mode, nu, gsp.maxk_threshold};
            RootResult r = solve_bracket_upper(f, 0., 100.);
            if (!r.ok) atomicOr(status_out, 4);
            maxk = sqrt(r.x) / rD;
            maxRrD = sqrt(pow(gsp.xvalue_accuracy, 1. / (1. - beta)) - 1.);
        }
        const double maxR = maxRrD * rD;
        if (beta <= 1.1) {
            stepk = kPi / maxR;
        } else {
            double R = pow(gsp.folding_threshold, 0.5 / (1. - beta)) * rD;
            if (R > maxR) R = maxR;
            // getHalfLightRadius (SBMoffat.cpp:247-258), of the truncated profile when truncated
            const double hlr = rD * sqrt(pow(1. - 0.5 * flux_factor, 1. / (1. - beta)) - 1.);
            R = fmax(R, gsp.stepk_minimum_hlr * hlr);
            stepk = kPi / R;
        }
        break;
      }
      case GSB_KOLMOGOROV: {
        // kolmogorov.py:163-226 (k0), :281-287; SBKolmogorov.cpp:117-121
        const double k0 = 2.992939911888651 / L.p[0];
        L.d[0] = 1. / k0;
        maxk = pow(-log(gsp.kvalue_accuracy), 0.6) * k0;
        stepk = kolm_stepk * k0;
        break;
      }
      case GSB_AIRY: {
        // airy.py:217-222, SBAiry.cpp:66-81, 332-356, 432-445
        const double lod = L.p[0], obs = L.p[1];
        const double D = 1. / lod;
        L.d[0] = 1. / (D * kPi);
        L.d[1] = L.flux / (kPi * (1. - obs * obs));
        L.d[2] = obs;
        L.d[3] = obs * obs;
        maxk = 2. * kPi / lod;
        double R = (obs == 0.) ? 1. / (gsp.folding_threshold * 0.5 * kPi * kPi)
                               : 1. / (gsp.folding_threshold * 0.5 * kPi * kPi * (1. - obs));
        R = fmax(R, gsp.stepk_minimum_hlr * 0.5348321477);
        stepk = kPi / R * D;
        break;
      }
      case GSB_BOX: {
        // box.py:100-106, SBBox.cpp:74-77
        const double w = L.p[0], hgt = L.p[1];
        L.d[0] = w / (2. * kPi);
        L.d[1] = hgt / (2. * kPi);
        maxk = 2. / (gsp.maxk_threshold * fmin(w, hgt));
        stepk = kPi / fmax(w, hgt);
        break;
      }
      case GSB_INTERPOLATED: {
        // SBInterpolatedImage.cpp:97-152: kscale = (N/2) / pi maps k to the k-image's sample
        // index, maxk1 = urange / uscale cuts where the x interpolant's transform is
        // negligible.  stepk holds the flux radius R and maxk the scanned maxk (image units),
        // which the host turns into the profile's world stepk / maxk.
        const int slot = L.table;
        const int xc = int(L.p[0]), kc = int(L.p[1]);
        if (slot < 0 || slot >= images.count) { atomicOr(status_out, 16); break; }
        if (xc < GSB_INTERP_DELTA || xc > GSB_INTERP_SINC || kc < GSB_INTERP_NEAREST ||
            kc > GSB_INTERP_LANCZOS) { atomicOr(status_out, 32); break; }
        // a Lanczos k interpolant: p[2] holds its coefficient block {n, conserve_dc, K_1..5};
        // n <= 3 (at most 7 taps per axis)
        const double* kt = reinterpret_cast<const double*>(__double_as_longlong(L.p[2]));
        if (kc == GSB_INTERP_LANCZOS && (kt == nullptr || kt[0] < 1. || kt[0] > 3.)) {
            atomicOr(status_out, 512);
            break;
        }
        const ImageSlot& I = images.slots[slot];
        if (xc != I.desc.x_interp) { atomicOr(status_out, 1024); break; }
        const int N = I.desc.N;
        L.d[0] = (N / 2) / kPi;
        // a Lanczos x interpolant's urange is its table's uMax (Lanczos::urange)
        L.d[1] = (xc == GSB_INTERP_LANCZOS ? I.desc.x_table[3] : interp_urange(xc, gsp.kvalue_accuracy)) /
                 (1. / (2. * kPi));
        L.d[5] = __longlong_as_double((long long)I.desc.x_table);
        L.d[2] = xc + 16 * kc;
        L.d[3] = __longlong_as_double(kc == GSB_INTERP_LANCZOS ? (long long)kt : 0LL);
        L.d[4] = N;
        L.d[6] = __longlong_as_double((long long)(images.k64 + I.k_offset));
        L.d[7] = __longlong_as_double((long long)(images.k32 + I.k_offset));
        stepk = images.info[2 * slot];
        maxk = images.info[2 * slot + 1];
        break;
      }
      default:
        atomicOr(status_out, 8);
    }
    info[2 * idx] = stepk;
    info[2 * idx + 1] = maxk;
}

}  // namespace

namespace {
__global__ void exp_tab_kernel(const double* x, double* y, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = exp_tab(x[i]);
}

__global__ void exp_tab256_kernel(const double* x, double* y, int n)
{
    __shared__ double etab[256];
    etab[threadIdx.x] = g_exp2_256[threadIdx.x];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = x[i] < -708. ? 0. : exp_tab256_core(x[i], etab);
}
}  // namespace

int exp_fp64(const double* d_x, double* d_y, int n, int table_size, cudaStream_t stream)
{
    if (n <= 0) return GSB_OK;
    if (table_size == 256)
        exp_tab256_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_x, d_y, n);
    else
        exp_tab_kernel<<<(n + 255) / 256, 256, 0, stream>>>(d_x, d_y, n);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

int ogata_init(DeviceState* st)
{
    {
        double tab[256];
        for (int j = 0; j < 256; ++j) tab[j] = (double)exp2l((long double)j / 256.L);
        GSB_CUDA_CHECK(cudaMemcpyToSymbol(g_exp2_256, tab, sizeof(tab)));
    }
    GSB_CUDA_CHECK(cudaMalloc(&st->d_status, sizeof(int)));
    GSB_CUDA_CHECK(cudaMalloc(&st->d_root, sizeof(double2) * kNroot));
    ogata_root_kernel<<<(unsigned)((kNroot + 255) / 256), 256>>>(st->d_root, kNroot);
    GSB_CUDA_CHECK(cudaGetLastError());
    long long total = 0;
    OgataTables og{};
    og.lev_min = kLevMin;
    og.lev_max = kLevMax;
    for (int lev = kLevMin; lev <= kLevMax; ++lev) {
        const double h = ldexp(1.0, -lev);
        const long long n = (long long)std::min(M_PI / h, 1e6);
        og.off[lev - kLevMin] = total;
        og.cnt[lev - kLevMin] = n;
        total += n;
    }
    GSB_CUDA_CHECK(cudaMalloc(&st->d_xw, sizeof(double2) * total));
    for (int lev = kLevMin; lev <= kLevMax; ++lev) {
        const long long n = og.cnt[lev - kLevMin];
        ogata_level_kernel<<<(unsigned)((n + 255) / 256), 256>>>(
            st->d_xw + og.off[lev - kLevMin], st->d_root, ldexp(1.0, -lev), n);
        GSB_CUDA_CHECK(cudaGetLastError());
    }
    GSB_CUDA_CHECK(cudaDeviceSynchronize());
    og.xw = st->d_xw;
    og.root = st->d_root;
    og.nroot = kNroot;
    st->og = og;
    return GSB_OK;
}

// Upper bound on the Sersic table length for these n values and GSParams.
static int sersic_stride(const double* h_n, int count, const gsb_gsparams* gsp)
{
    double nmax = 0.;
    for (int i = 0; i < count; ++i) nmax = std::max(nmax, h_n[i]);
    const double kderiv6 = std::exp(std::lgamma(8. * nmax) - std::lgamma(2. * nmax)) / 2304.;
    const double kmin = std::pow(gsp->kvalue_accuracy / kderiv6, 1. / 6.);
    const double dlogk = gsp->table_spacing * std::sqrt(std::sqrt(gsp->kvalue_accuracy / 10.));
    const double span = std::log(500.) - (std::log(kmin) - 0.001);
    return int(span / dlogk) + 4;
}

int sersic_tables_build(gsb_tables* t, const double* h_n, const double* h_trunc, int count,
                        const gsb_gsparams* gsp, bool with_dn, cudaStream_t stream)
{
    DeviceState* st = device_state();
    if (!st->ready) return set_error(GSB_ERR_INVALID, "gsb_init has not been called");
    for (int i = 0; i < count; ++i) {
        if (!(h_n[i] >= 0.3 && h_n[i] <= 6.2))
            return set_error(GSB_ERR_INVALID, "Sersic index out of range [0.3, 6.2]");
        if (h_trunc && !(h_trunc[i] >= 0.))
            return set_error(GSB_ERR_INVALID, "Sersic truncation radius must be >= 0");
    }
    if (count <= 0) { t->count = 0; return GSB_OK; }
    bool has_trunc = false;
    for (int i = 0; h_trunc && i < count; ++i) has_trunc |= h_trunc[i] > 0.;
    if (has_trunc && with_dn)
        return set_error(GSB_ERR_UNSUPPORTED, "n-derivative tables of truncated Sersic profiles are not built");
    const int stride = sersic_stride(h_n, count, gsp);
    if ((size_t)count > t->cap_slots || (size_t)count * stride > t->cap_nodes) {
        cudaFree(t->d_header); cudaFree(t->d_node); cudaFree(t->d_val); cudaFree(t->d_scan);
        cudaFree(t->d_n); cudaFree(t->d_status);
        t->d_header = nullptr; t->d_node = nullptr; t->d_val = nullptr; t->d_scan = nullptr;
        t->d_n = nullptr; t->d_status = nullptr;
        t->cap_slots = std::max<size_t>(count, t->cap_slots);
        t->cap_nodes = std::max<size_t>((size_t)count * stride, t->cap_nodes);
        GSB_CUDA_CHECK(cudaMalloc(&t->d_header, sizeof(double) * kSersicHeader * t->cap_slots));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_node, sizeof(double4) * t->cap_nodes));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_val, sizeof(double) * t->cap_nodes));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_scan, sizeof(SersicScan) * t->cap_slots));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_n, sizeof(double) * t->cap_slots));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_status, sizeof(int) * (1 + kMaxRounds)));
    }
    if (with_dn && ((size_t)count > t->cap_dn_slots || (size_t)count * stride > t->cap_dn_nodes)) {
        cudaFree(t->d_dheader); cudaFree(t->d_dnode); cudaFree(t->d_dval);
        t->d_dheader = nullptr; t->d_dnode = nullptr; t->d_dval = nullptr;
        t->cap_dn_slots = std::max<size_t>(count, t->cap_dn_slots);
        t->cap_dn_nodes = std::max<size_t>((size_t)count * stride, t->cap_dn_nodes);
        GSB_CUDA_CHECK(cudaMalloc(&t->d_dheader, sizeof(double) * kSersicDHeader * t->cap_dn_slots));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_dnode, sizeof(double4) * t->cap_dn_nodes));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_dval, sizeof(double) * t->cap_dn_nodes));
    }
    t->has_dn = with_dn;
    double* dheader = with_dn ? t->d_dheader : nullptr;
    double4* dnode = with_dn ? t->d_dnode : nullptr;
    double* dval = with_dn ? t->d_dval : nullptr;
    t->count = count;
    t->stride = stride;
    double* d_n = t->d_n;
    int* d_status = t->d_status;
    GSB_CUDA_CHECK(cudaMemcpyAsync(d_n, h_n, sizeof(double) * count, cudaMemcpyHostToDevice, stream));
    double* d_trunc = nullptr;
    if (has_trunc) {
        if ((size_t)count > t->cap_trunc) {
            cudaFree(t->d_trunc);
            t->d_trunc = nullptr;
            t->cap_trunc = count;
            GSB_CUDA_CHECK(cudaMalloc(&t->d_trunc, sizeof(double) * t->cap_trunc));
        }
        d_trunc = t->d_trunc;
        GSB_CUDA_CHECK(cudaMemcpyAsync(d_trunc, h_trunc, sizeof(double) * count, cudaMemcpyHostToDevice, stream));
    }
    if ((stride + kTableRound - 1) / kTableRound > kMaxRounds) return set_error(GSB_ERR_UNSUPPORTED, "Sersic table too long");
    const size_t fsm = sizeof(double) * 4 * (size_t)stride;
    if (fsm > 227 * 1024) return set_error(GSB_ERR_UNSUPPORTED, "Sersic table too long");
    if (fsm > 48 * 1024)
        GSB_CUDA_CHECK(cudaFuncSetAttribute(sersic_finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(std::min<size_t>(fsm, 227 * 1024))));
    // the device part of the build: set-up, the rounds of nodes and their stopping scans, the
    // finalisation (no host synchronisation inside)
    auto enqueue = [&](cudaStream_t stream) -> int {
        // d_status[0]: convergence status; d_status[1 + r]: some table still needs nodes after round r
        GSB_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int) * (1 + kMaxRounds), stream));
        sersic_setup_kernel<<<(count + 127) / 128, 128, 0, stream>>>(d_n, d_trunc, count, *gsp, t->d_header, stride,
                                                                     dheader);
        GSB_CUDA_CHECK(cudaGetLastError());
        sersic_scan_init_kernel<<<(count + 127) / 128, 128, 0, stream>>>(t->d_header, count, static_cast<SersicScan*>(t->d_scan));
        GSB_CUDA_CHECK(cudaGetLastError());
        // Rounds of kRound ln k nodes: integrate, then advance each table's stopping scan.
        constexpr int kRound = kTableRound;
        const int threads = 256;
        for (int i0 = 0, r = 0; i0 < stride; i0 += kRound, ++r) {
            const int* prev_live = r > 0 ? d_status + r : nullptr;
            const long long nwarps = (long long)count * ((kRound + 1) / 2);
            const long long blocks = (nwarps * 32 + threads - 1) / threads;
            if (with_dn)
                sersic_nodes_pair_kernel<true><<<(unsigned)blocks, threads, 0, stream>>>(
                    t->d_header, count, i0, kRound, *gsp, st->og, static_cast<const SersicScan*>(t->d_scan),
                    t->d_val, stride, prev_live, d_status, dheader, dval);
            else
                sersic_nodes_pair_kernel<false><<<(unsigned)blocks, threads, 0, stream>>>(
                    t->d_header, count, i0, kRound, *gsp, st->og, static_cast<const SersicScan*>(t->d_scan),
                    t->d_val, stride, prev_live, d_status, nullptr, nullptr);
            GSB_CUDA_CHECK(cudaGetLastError());
            if (has_trunc) {
                const long long tw = (long long)count * kRound;
                sersic_trunc_nodes_kernel<<<(unsigned)((tw * 32 + threads - 1) / threads), threads, 0, stream>>>(
                    t->d_header, count, i0, kRound, st->og, static_cast<const SersicScan*>(t->d_scan), t->d_val, stride,
                    prev_live, d_status);
                GSB_CUDA_CHECK(cudaGetLastError());
            }
            sersic_scan_kernel<<<(count + 63) / 64, 64, 0, stream>>>(t->d_header, count, stride, i0, kRound,
                                                                     *gsp, t->d_val, t->d_node, static_cast<SersicScan*>(t->d_scan),
                                                                     dval, dnode, prev_live, d_status + 1 + r);
            GSB_CUDA_CHECK(cudaGetLastError());
        }
        sersic_finalize_kernel<<<count, 32, fsm, stream>>>(t->d_header, count, stride, *gsp,
                                                            static_cast<const SersicScan*>(t->d_scan), t->d_node,
                                                            dnode, dheader);
        GSB_CUDA_CHECK(cudaGetLastError());
        return GSB_OK;
    };
    // The launches are captured once as a CUDA graph and replayed while the build's shape is
    // unchanged (table count, node stride, flags, GSParams and buffers: the captured launches
    // hold them); the captured early-exit rounds then cost a graph node each instead of a launch.
    struct Key {
        int count, stride, with_dn, has_trunc;
        gsb_gsparams gsp;
        const void* ptr[12];
    } key;
    std::memset(&key, 0, sizeof(key));
    key.count = count;
    key.stride = stride;
    key.with_dn = with_dn;
    key.has_trunc = has_trunc;
    key.gsp = *gsp;
    const void* ptrs[12] = {t->d_header, t->d_node, t->d_val, t->d_scan, d_n, d_status, d_trunc, dheader,
                            dnode, dval, st->og.xw, st->og.root};
    for (int k = 0; k < 12; ++k) key.ptr[k] = ptrs[k];
    static_assert(sizeof(Key) <= sizeof(t->sersic_key), "graph key too large");
    if (!(t->sersic_exec && std::memcmp(t->sersic_key, &key, sizeof(key)) == 0)) {
        if (t->sersic_exec) { cudaGraphExecDestroy(t->sersic_exec); t->sersic_exec = nullptr; }
        // captured on a private stream (the caller's may be the legacy default stream, which
        // cannot be captured); capturing runs nothing
        if (!t->capture_stream) GSB_CUDA_CHECK(cudaStreamCreateWithFlags(&t->capture_stream, cudaStreamNonBlocking));
        GSB_CUDA_CHECK(cudaStreamBeginCapture(t->capture_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue(t->capture_stream);
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(t->capture_stream, &graph);
        if (rc || ce != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return rc ? rc : set_error(GSB_ERR_CUDA, std::string("table-build capture: ") + cudaGetErrorString(ce));
        }
        const cudaError_t ie = cudaGraphInstantiate(&t->sersic_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            t->sersic_exec = nullptr;
            return set_error(GSB_ERR_CUDA, std::string("table-build graph: ") + cudaGetErrorString(ie));
        }
        std::memcpy(t->sersic_key, &key, sizeof(key));
    }
    GSB_CUDA_CHECK(cudaGraphLaunch(t->sersic_exec, stream));
    int h_status = 0;
    GSB_CUDA_CHECK(cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status) return set_error(GSB_ERR_NUMERIC, "Sersic Hankel transform did not converge");
    return GSB_OK;
}

int sersic_truncation(int count, const double* h_in, double* h_out, cudaStream_t stream)
{
    if (count <= 0) return GSB_OK;
    double *d_in = nullptr, *d_out = nullptr;
    int* d_status = nullptr;
    GSB_CUDA_CHECK(cudaMallocAsync(&d_in, sizeof(double) * 4 * count, stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_out, sizeof(double) * 2 * count, stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_status, sizeof(int), stream));
    GSB_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(d_in, h_in, sizeof(double) * 4 * count, cudaMemcpyHostToDevice, stream));
    sersic_truncation_kernel<<<(count + 127) / 128, 128, 0, stream>>>(d_in, count, d_out, d_status);
    GSB_CUDA_CHECK(cudaGetLastError());
    int h_status = 0;
    GSB_CUDA_CHECK(cudaMemcpyAsync(h_out, d_out, sizeof(double) * 2 * count, cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    cudaFreeAsync(d_in, stream);
    cudaFreeAsync(d_out, stream);
    cudaFreeAsync(d_status, stream);
    if (h_status) return set_error(GSB_ERR_NUMERIC, "truncated Sersic scale radius root find did not converge");
    return GSB_OK;
}

// The reference's k grid of SBMoffat::setupFT: k = 0, dk, 2 dk, ... as a running sum, k < 50.
static std::vector<double> moffat_kgrid(const gsb_gsparams* gsp)
{
    const double dk = gsp->table_spacing * std::sqrt(std::sqrt(gsp->kvalue_accuracy / 10.));
    std::vector<double> k;
    for (double x = 0.; x < 50.; x += dk) k.push_back(x);
    return k;
}

int moffat_tables_build(gsb_tables* t, const double* h_beta, const double* h_trunc, int count,
                        const gsb_gsparams* gsp, cudaStream_t stream)
{
    DeviceState* st = device_state();
    if (!st->ready) return set_error(GSB_ERR_INVALID, "gsb_init has not been called");
    for (int i = 0; i < count; ++i) {
        if (!(h_trunc[i] > 0.) || !std::isfinite(h_trunc[i]))
            return set_error(GSB_ERR_INVALID, "Moffat table needs trunc / scale_radius > 0");
        if (!(h_beta[i] > 0.) || h_beta[i] == 1. || !std::isfinite(h_beta[i]))
            return set_error(GSB_ERR_INVALID, "truncated Moffat beta must be > 0 and != 1 (at beta = 1 the "
                                              "flux normalisation 2 (beta - 1) / (1 - (1 + t^2)^(1 - beta)) is 0/0)");
    }
    if (count <= 0) { t->moffat_count = 0; return GSB_OK; }
    if (!(gsp->kvalue_accuracy > 0.) || !(gsp->table_spacing > 0.))
        return set_error(GSB_ERR_INVALID, "kvalue_accuracy and table_spacing must be > 0");
    const std::vector<double> kg = moffat_kgrid(gsp);
    const int ncand = int(kg.size());
    const size_t fsm = sizeof(double) * 4 * (size_t)ncand;
    if (fsm > 227 * 1024)
        return set_error(GSB_ERR_UNSUPPORTED, "truncated Moffat table too long for this kvalue_accuracy / "
                                              "table_spacing (more than 7264 nodes)");
    if ((size_t)count > t->cap_mslots || (size_t)count * ncand > t->cap_mnodes || (size_t)ncand > t->cap_mk) {
        cudaFree(t->d_mheader); cudaFree(t->d_mnode); cudaFree(t->d_mval); cudaFree(t->d_mk); cudaFree(t->d_mstatus);
        t->d_mheader = nullptr; t->d_mnode = nullptr; t->d_mval = nullptr; t->d_mk = nullptr; t->d_mstatus = nullptr;
        t->cap_mslots = std::max<size_t>(count, t->cap_mslots);
        t->cap_mnodes = std::max<size_t>((size_t)count * ncand, t->cap_mnodes);
        t->cap_mk = std::max<size_t>(ncand, t->cap_mk);
        GSB_CUDA_CHECK(cudaMalloc(&t->d_mheader, sizeof(double) * kMoffatHeader * t->cap_mslots));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_mnode, sizeof(double4) * t->cap_mnodes));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_mval, sizeof(double) * t->cap_mnodes));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_mk, sizeof(double) * t->cap_mk));
        GSB_CUDA_CHECK(cudaMalloc(&t->d_mstatus, sizeof(int)));
    }
    t->moffat_count = count;
    t->moffat_stride = ncand;
    // slot headers: (beta, trunc / rD, dk) from the host, the rest written on the device
    std::vector<double> hh((size_t)kMoffatHeader * count, 0.);
    for (int i = 0; i < count; ++i) {
        hh[(size_t)i * kMoffatHeader + kMH_BETA] = h_beta[i];
        hh[(size_t)i * kMoffatHeader + kMH_TRUNC] = h_trunc[i];
        hh[(size_t)i * kMoffatHeader + kMH_DK] = ncand > 1 ? kg[1] : 0.;
    }
    GSB_CUDA_CHECK(cudaMemcpyAsync(t->d_mheader, hh.data(), sizeof(double) * hh.size(), cudaMemcpyHostToDevice,
                                   stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(t->d_mk, kg.data(), sizeof(double) * ncand, cudaMemcpyHostToDevice, stream));
    GSB_CUDA_CHECK(cudaMemsetAsync(t->d_mstatus, 0, sizeof(int), stream));
    moffat_setup_kernel<<<(count + 127) / 128, 128, 0, stream>>>(count, t->d_mheader);
    GSB_CUDA_CHECK(cudaGetLastError());
    const int threads = 256;
    const long long nwarps = (long long)count * ncand;
    moffat_nodes_kernel<<<(unsigned)((nwarps * 32 + threads - 1) / threads), threads, 0, stream>>>(
        t->d_mheader, count, t->d_mk, ncand, st->og, t->d_mval, t->d_mstatus);
    GSB_CUDA_CHECK(cudaGetLastError());
    if (fsm > 48 * 1024)
        GSB_CUDA_CHECK(cudaFuncSetAttribute(moffat_finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(fsm)));
    moffat_finalize_kernel<<<count, 32, fsm, stream>>>(t->d_mheader, count, t->d_mk, ncand, *gsp, t->d_mval,
                                                       t->d_mnode);
    GSB_CUDA_CHECK(cudaGetLastError());
    int h_status = 0;
    GSB_CUDA_CHECK(cudaMemcpyAsync(&h_status, t->d_mstatus, sizeof(int), cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status) return set_error(GSB_ERR_NUMERIC, "truncated Moffat Hankel transform ran out of J0 zeros");
    return GSB_OK;
}

int moffat_scale_radius(int count, const double* h_in, double* h_out, cudaStream_t stream)
{
    if (count <= 0) return GSB_OK;
    double *d_in = nullptr, *d_out = nullptr;
    int* d_status = nullptr;
    GSB_CUDA_CHECK(cudaMallocAsync(&d_in, sizeof(double) * 3 * count, stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_out, sizeof(double) * count, stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_status, sizeof(int), stream));
    GSB_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(d_in, h_in, sizeof(double) * 3 * count, cudaMemcpyHostToDevice, stream));
    moffat_scale_radius_kernel<<<(count + 127) / 128, 128, 0, stream>>>(d_in, count, d_out, d_status);
    GSB_CUDA_CHECK(cudaGetLastError());
    int h_status = 0;
    GSB_CUDA_CHECK(cudaMemcpyAsync(h_out, d_out, sizeof(double) * count, cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    cudaFreeAsync(d_in, stream);
    cudaFreeAsync(d_out, stream);
    cudaFreeAsync(d_status, stream);
    if (h_status) return set_error(GSB_ERR_NUMERIC, "Solve error: Moffat scale radius root find did not converge");
    return GSB_OK;
}

// The Kolmogorov radial spline of each device (its GSParams are those of the stepk cached in
// the device state).
namespace {
struct KolmRadial {
    double4* nodes = nullptr;
    int n = 0, cap = 0;
};
KolmRadial g_kolm_radial[64];
}  // namespace

static int kolmogorov_build(const gsb_gsparams* gsp, cudaStream_t stream)
{
    DeviceState* st = device_state();
    int dev = 0;
    cudaGetDevice(&dev);
    KolmRadial& kr = g_kolm_radial[dev & 63];
    const double key[13] = {double(gsp->minimum_fft_size), double(gsp->maximum_fft_size),
                            gsp->folding_threshold, gsp->stepk_minimum_hlr, gsp->maxk_threshold,
                            gsp->kvalue_accuracy, gsp->xvalue_accuracy, gsp->table_spacing,
                            gsp->realspace_relerr, gsp->realspace_abserr, gsp->integration_relerr,
                            gsp->integration_abserr, gsp->shoot_accuracy};
    if (st->kolm_valid && std::equal(key, key + 13, st->kolm_key)) return GSB_OK;
    const double dlogr = gsp->table_spacing * std::sqrt(std::sqrt(gsp->xvalue_accuracy / 10.));
    int ncand = 0;
    for (double logr = -3.; logr < std::log(1.e4); logr += dlogr) ++ncand;
    if (ncand + 1 > kr.cap) {
        cudaFree(kr.nodes);
        kr.nodes = nullptr;
        kr.cap = 0;
        GSB_CUDA_CHECK(cudaMalloc(&kr.nodes, sizeof(double4) * (ncand + 1)));
        kr.cap = ncand + 1;
    }
    double* d_vals = nullptr;
    int* d_status = nullptr;
    double* d_out = nullptr;
    double* d_scratch = nullptr;
    GSB_CUDA_CHECK(cudaMallocAsync(&d_vals, sizeof(double) * ncand, stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_status, sizeof(int), stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_out, sizeof(double) * 2, stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_scratch, sizeof(double) * 4 * (ncand + 1), stream));
    GSB_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), stream));
    kolmogorov_nodes_kernel<<<(ncand * 32 + 255) / 256, 256, 0, stream>>>(ncand, dlogr, *gsp, st->og,
                                                                          d_vals, d_status);
    GSB_CUDA_CHECK(cudaGetLastError());
    kolmogorov_finalize_kernel<<<1, 1, 0, stream>>>(ncand, dlogr, *gsp, d_vals, d_out, kr.nodes, d_scratch);
    GSB_CUDA_CHECK(cudaGetLastError());
    double h_out[2] = {0., 0.};
    int h_status = 0;
    GSB_CUDA_CHECK(cudaMemcpyAsync(h_out, d_out, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaFreeAsync(d_vals, stream));
    GSB_CUDA_CHECK(cudaFreeAsync(d_status, stream));
    GSB_CUDA_CHECK(cudaFreeAsync(d_out, stream));
    GSB_CUDA_CHECK(cudaFreeAsync(d_scratch, stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status) return set_error(GSB_ERR_NUMERIC, "Kolmogorov Hankel transform did not converge");
    std::copy(key, key + 13, st->kolm_key);
    st->kolm_stepk = h_out[0];
    kr.n = int(h_out[1]);
    st->kolm_valid = true;
    return GSB_OK;
}

int kolmogorov_stepk(const gsb_gsparams* gsp, cudaStream_t stream, double* out)
{
    const int rc = kolmogorov_build(gsp, stream);
    if (rc) return rc;
    *out = device_state()->kolm_stepk;
    return GSB_OK;
}

// The radial spline nodes (r, f, y2, 0) of KolmogorovInfo for these GSParams (gsb_real.cu).
int kolmogorov_radial(const gsb_gsparams* gsp, cudaStream_t stream, const double4** nodes, int* n)
{
    const int rc = kolmogorov_build(gsp, stream);
    if (rc) return rc;
    int dev = 0;
    cudaGetDevice(&dev);
    *nodes = g_kolm_radial[dev & 63].nodes;
    *n = g_kolm_radial[dev & 63].n;
    return GSB_OK;
}

int prepare_leaves(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp, gsb_leaf* d_leaves,
                   const gsb_tables* t, double* d_info, cudaStream_t stream)
{
    DeviceState* st = device_state();
    if (!st->ready) return set_error(GSB_ERR_INVALID, "gsb_init has not been called");
    bool need_kolm = false, need_sersic = false, need_images = false;
    for (int l = 0; l < tpl->n_leaves; ++l) {
        if (tpl->leaf_type[l] == GSB_KOLMOGOROV) need_kolm = true;
        if (tpl->leaf_type[l] == GSB_SERSIC) need_sersic = true;
        if (tpl->leaf_type[l] == GSB_INTERPOLATED) need_images = true;
    }
    if (need_sersic && (!t || t->count == 0))
        return set_error(GSB_ERR_INVALID, "Sersic leaves need built FT tables");
    if (need_images && (!t || t->n_images == 0))
        return set_error(GSB_ERR_INVALID, "InterpolatedImage leaves need built image slots");
    ImageRefs images{};
    if (t) images = ImageRefs{t->d_images, t->d_image_info, t->d_k64, t->d_k32, t->n_images};
    MoffatRefs moffat{};
    if (t) moffat = MoffatRefs{t->d_mheader, t->d_mnode, t->moffat_count, t->moffat_stride};
    double kolm = 0.;
    if (need_kolm) {
        const int rc = kolmogorov_stepk(gsp, stream, &kolm);
        if (rc) return rc;
    }
    int* d_status = st->d_status;
    GSB_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), stream));
    const long long n = (long long)n_stamps * tpl->n_leaves;
    if (n > 0) {
        prepare_leaves_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(
            *tpl, n_stamps, *gsp, d_leaves, t ? t->d_header : nullptr, moffat, kolm, images, d_info, d_status);
        GSB_CUDA_CHECK(cudaGetLastError());
    }
    int h_status = 0;
    GSB_CUDA_CHECK(cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h_status & 8) return set_error(GSB_ERR_INVALID, "unknown leaf type");
    if (h_status & 16) return set_error(GSB_ERR_INVALID, "InterpolatedImage leaf names no built image slot");
    if (h_status & 32) return set_error(GSB_ERR_UNSUPPORTED, "interpolant not built (x: Delta, Nearest, "
                                                             "Linear, Cubic, Quintic, Lanczos; k: the same "
                                                             "but Delta)");
    if (h_status & 512) return set_error(GSB_ERR_INVALID, "a Lanczos k interpolant needs its coefficient "
                                                          "block in p[2] (n <= 3)");
    if (h_status & 1024) return set_error(GSB_ERR_INVALID, "InterpolatedImage leaf's x interpolant differs "
                                                           "from its image slot's");
    if (h_status & 2) return set_error(GSB_ERR_NUMERIC, "Sersic radius root finding failed");
    if (h_status & 4) return set_error(GSB_ERR_NUMERIC, "Moffat maxk root finding failed");
    if (h_status & 64) return set_error(GSB_ERR_INVALID, "truncated Moffat leaf names no built Moffat table slot");
    if (h_status & 128) return set_error(GSB_ERR_INVALID, "truncated Moffat leaf's table slot was built for "
                                                          "another (beta, trunc / scale_radius)");
    if (h_status & 256) return set_error(GSB_ERR_NUMERIC, "truncated Moffat table is empty");
    return GSB_OK;
}

}  // namespace gsb
