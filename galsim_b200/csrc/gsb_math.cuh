// FP64 device mathematics for the sizing / table stage.
//
// Everything here runs on the GPU in double precision.  The algorithms are written from
// their published descriptions; the reference's own implementations are cited where the
// behaviour (brackets, tolerances, stopping rules) must match.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace gsb {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------
// Regularised lower incomplete gamma P(a, x) = gamma(a, x) / Gamma(a).
// Reference: math::gamma_p (src/math/Gamma.cpp:49-70, SLATEC dgamit).  Here: the power
// series  P = x^a e^-x / Gamma(a+1) * sum_k x^k / ((a+1)...(a+k))  for x < a + 1 and the
// Legendre continued fraction for Q = 1 - P (evaluated with the modified Lentz method)
// otherwise (Abramowitz & Stegun 6.5.29 and 6.5.31).
// ---------------------------------------------------------------------------------------
__device__ inline double gamma_p(double a, double x)
{
    if (x <= 0.) return 0.;
    const double lpre = -x + a * log(x) - lgamma(a);
    if (x < a + 1.) {
        double term = 1. / a, sum = term;
        for (int k = 1; k < 1000; ++k) {
            term *= x / (a + k);
            sum += term;
            if (fabs(term) < fabs(sum) * 1e-17) break;
        }
        return sum * exp(lpre);
    } else {
        const double tiny = 1e-300;
        double b = x + 1. - a;
        double c = 1. / tiny;
        double d = 1. / b;
        double h = d;
        for (int i = 1; i < 1000; ++i) {
            const double an = -i * (i - a);
            b += 2.;
            d = an * d + b;
            if (fabs(d) < tiny) d = tiny;
            c = b + an / c;
            if (fabs(c) < tiny) c = tiny;
            d = 1. / d;
            const double del = d * c;
            h *= del;
            if (fabs(del - 1.) < 1e-16) break;
        }
        return 1. - exp(lpre) * h;
    }
}

// ---------------------------------------------------------------------------------------
// FP64 exponential for the Hankel quadrature, by the table-driven method of P. T. P. Tang,
// "Table-driven implementation of the exponential function in IEEE floating-point arithmetic",
// ACM TOMS 15 (1989) 144-157:  x = (32 m + j) ln2/32 + r with |r| <= ln2/64 (the reduction in
// two FMA steps with ln2/32 split into a double and its remainder), exp(x) = 2^m 2^(j/32) p(r),
// p the degree-6 Taylor polynomial of e^r (truncation < 4e-18 relative), 2^(j/32) correctly
// rounded.  Within ~2 ulp of exp for -708 <= x <= 709; 0 below -708 (the terms that reach it
// are far below the quadrature's stopping threshold).
// ---------------------------------------------------------------------------------------
__device__ const double kExp2Tab[32] = {
    1.0, 1.0218971486541166, 1.0442737824274138, 1.0671404006768237, 1.0905077326652577,
    1.1143867425958924, 1.1387886347566916, 1.1637248587775775, 1.189207115002721,
    1.215247359980469, 1.241857812073484, 1.2690509571917332, 1.2968395546510096,
    1.3252366431597413, 1.3542555469368927, 1.383909881963832, 1.4142135623730951,
    1.4451808069770467, 1.4768261459394993, 1.5091644275934228, 1.5422108254079407,
    1.5759808451078865, 1.6104903319492543, 1.645755478153965, 1.681792830507429,
    1.718619298122478, 1.7562521603732995, 1.7947090750031072, 1.8340080864093424,
    1.8741676341103, 1.9152065613971474, 1.9571441241754002};

// The exponential's body for -708 <= x <= 709 (no range test); `tab` is kExp2Tab or a copy of
// it (in shared memory, for kernels that evaluate many exponentials per thread).
__device__ __forceinline__ double exp_tab_core(double x, const double* tab = kExp2Tab)
{
    // n = rint(x 32/ln2) without a rounding or conversion instruction: adding 1.5 * 2^52 to the
    // (rounded) product leaves n, rounded to nearest-even as rint does, in the low mantissa bits
    // (|n| < 2^31), and subtracting it back gives n as a double exactly.
    const double kShift = 6755399441055744.0;               // 1.5 * 2^52
    const double s = __dadd_rn(__dmul_rn(x, 46.16624130844683), kShift);   // 32 / ln2
    const int n = __double2loint(s);
    const double t = s - kShift;
    double r = fma(-t, 0.02166084939249829, x);              // ln2/32, leading double
    r = fma(-t, 7.247021293269686e-19, r);                   // ln2/32, remainder
    const int j = n & 31;
    const int m = n >> 5;
    double p = fma(r, 1. / 720., 1. / 120.);
    p = fma(p, r, 1. / 24.);
    p = fma(p, r, 1. / 6.);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.);
    p = fma(p, r, 1.);
    const double v = tab[j] * p;
    return __hiloint2double(__double2hiint(v) + (m << 20), __double2loint(v));
}

__device__ __forceinline__ double exp_tab(double x)
{
    if (x < -708.) return 0.;
    return exp_tab_core(x);
}

// exp(x) for x <= 0 without a branch: arguments below -708 give exp(-708) ~ 3e-308 instead
// of 0 (the quadrature's terms that reach them are far below its stopping threshold).
__device__ __forceinline__ double exp_tab_neg(double x, const double* tab = kExp2Tab)
{
    return exp_tab_core(fmax(x, -708.), tab);
}

// ---------------------------------------------------------------------------------------
// Digamma psi(x) = d ln Gamma / dx for x > 0: the recurrence psi(x) = psi(x + 1) - 1/x
// (A&S 6.3.5) up to x >= 10, then the asymptotic series
// psi(x) ~ ln x - 1/(2x) - sum_k B_2k / (2k x^2k)  (A&S 6.3.18), five terms.
// ---------------------------------------------------------------------------------------
__device__ inline double digamma(double x)
{
    double r = 0.;
    while (x < 10.) { r -= 1. / x; x += 1.; }
    const double ix2 = 1. / (x * x);
    const double series = ix2 * (1. / 12. - ix2 * (1. / 120. - ix2 * (1. / 252. - ix2 * (1. / 240. - ix2 * (1. / 132.)))));
    return r + log(x) - 0.5 / x - series;
}

// dP(a, x)/da by a central difference of gamma_p in FP64 (relative step 1e-5): P is smooth
// in a and accurate to ~1e-16, so the difference is good to ~1e-10.
__device__ inline double gamma_p_da(double a, double x)
{
    const double h = 1e-5 * a;
    return (gamma_p(a + h, x) - gamma_p(a - h, x)) / (2. * h);
}

// ---------------------------------------------------------------------------------------
// Brent's root finder with the reference's bracket expansion rules
// (include/galsim/Solve.h: defaultTolerance 1e-7, defaultMaxSteps 40, bracket1 :217-232,
// bracket1WithLimit :264-326, zbrent :385-447).  Brent's method itself follows the
// published algorithm (R. P. Brent, "Algorithms for Minimization without Derivatives",
// 1973, ch. 4).  `ok` is cleared when a bracket or the iteration fails.
// ---------------------------------------------------------------------------------------
struct RootResult { double x; bool ok; };

template <class F>
__device__ RootResult brent_root(const F& f, double a, double b, double fa, double fb)
{
    const double xtol = 1e-7;
    const int max_steps = 40;
    if ((fa > 0. && fb > 0.) || (fa < 0. && fb < 0.)) return {b, false};
    double c = b, fc = fb, d = b - a, e = d;
    for (int it = 0; it <= max_steps; ++it) {
        if ((fb > 0. && fc > 0.) || (fb < 0. && fc < 0.)) { c = a; fc = fa; e = d = b - a; }
        if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
        const double tol1 = 2. * 2.220446049250313e-16 * fabs(b) + 0.5 * xtol;
        const double xm = 0.5 * (c - b);
        if (fabs(xm) <= tol1 || fb == 0.) return {b, true};
        if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
            const double s = fb / fa;
            double p, q;
            if (a == c) { p = 2. * xm * s; q = 1. - s; }
            else {
                const double qq = fa / fc, r = fb / fc;
                p = s * (2. * xm * qq * (qq - r) - (b - a) * (r - 1.));
                q = (qq - 1.) * (r - 1.) * (s - 1.);
            }
            if (p > 0.) q = -q;
            p = fabs(p);
            const double min1 = 3. * xm * q - fabs(tol1 * q), min2 = fabs(e * q);
            if (2. * p < fmin(min1, min2)) { e = d; d = p / q; }
            else { d = xm; e = d; }
        } else { d = xm; e = d; }
        a = b; fa = fb;
        if (fabs(d) > tol1) b += d;
        else b += (xm >= 0. ? fabs(tol1) : -fabs(tol1));
        fb = f(b);
    }
    return {b, false};
}

// Expand the upper bound geometrically until the root is bracketed, then solve.
template <class F>
__device__ RootResult solve_bracket_upper(const F& f, double lo, double hi)
{
    double flo = f(lo), fhi = f(hi);
    double delta = hi - lo;
    int j = 1;
    for (; j < 40; ++j) {
        if (flo * fhi <= 0.) break;
        lo = hi; flo = fhi;
        delta *= 2.;
        hi += delta;
        fhi = f(hi);
    }
    if (flo * fhi > 0.) return {hi, false};
    return brent_root(f, lo, hi, flo, fhi);
}

// Expand the lower bound towards `limit` (never reaching it) until bracketed, then solve.
template <class F>
__device__ RootResult solve_bracket_lower_limit(const F& f, double lo, double hi, double limit)
{
    double flo = f(lo), fhi = f(hi);
    // Expansion moves `b` (here: lo) towards c = limit, keeping a = the previous point.
    double a = hi, fa = fhi, b = lo, fb = flo;
    int j = 1;
    for (; j < 40; ++j) {
        if (fa * fb <= 0.) break;
        const double bma = b - a, cmb = limit - b;
        a = b; fa = fb;
        b = (2. * limit / cmb + a / bma) / (2. / cmb + 1. / bma);
        fb = f(b);
    }
    if (fa * fb > 0.) return {b, false};
    // The solver is given (lBound, uBound) = (b, a) in the reference's order.
    return brent_root(f, b, a, fb, fa);
}

// ---------------------------------------------------------------------------------------
// Zeros of J0 and the Ogata (2005) quadrature nodes for Hankel transforms of order 0.
// j_{0,s}: McMahon's asymptotic expansion (A&S 9.5.12) refined by Newton steps on J0
// (J0' = -J1).  Node/weight formulas follow Ogata, Publ. RIMS 41 (2005) 949, as used by the
// reference's HankelIntegrator (src/math/Hankel.cpp:79-141):
//   xi = j_{0,s}/pi,  t = h xi,  x = pi/h psi(t),  psi(t) = t tanh(pi/2 sinh t)
//   w  = Y0(pi xi)/J1(pi xi) * pi x J0(x) psi'(t)
// ---------------------------------------------------------------------------------------
__device__ inline double bessel_j0_zero(long s)
{
    const double beta = (s - 0.25) * kPi;
    const double b8 = 8. * beta, ib = 1. / b8, ib2 = ib * ib;
    double x = beta + ib * (1. + ib2 * (-124. / 3. + ib2 * (120928. / 15.)));
    for (int it = 0; it < 4; ++it) x += j0(x) / j1(x);
    return x;
}

__device__ inline double ogata_psi(double t)
{ return t * tanh(0.5 * kPi * sinh(t)); }

__device__ inline double ogata_dpsi(double t)
{
    const double c = cosh(0.5 * kPi * sinh(t));
    return t * 0.5 * kPi * cosh(t) / (c * c) + ogata_psi(t) / t;
}

// ---------------------------------------------------------------------------------------
// c_nu x^nu K_nu(x) with c_nu = 2^(1-nu) / Gamma(nu), so that the value at x = 0 is 1.
// K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt  (DLMF 10.32.9); the integrand is entire
// and decays double-exponentially, so the trapezoid rule with step tau converges with
// error ~ exp(-pi^2 / (2 tau)).  Used for the Moffat Fourier transform
// (src/SBMoffat.cpp:296-345: kV = K_{beta-1}(k) k^{beta-1} * 4 / (Gamma(beta-1) 2^beta)).
// ---------------------------------------------------------------------------------------
__device__ inline double moffat_kv_fp64(double nu, double x)
{
    if (x <= 0.) return 1.;
    const double tau = 0.125;
    const double lognorm = (1. - nu) * log(2.) - lgamma(nu) + nu * log(x);
    // 0.5 * tau * f(0) + tau * sum_{j>=1} f(j tau), terms until negligible
    double sum = 0.5 * exp(lognorm - x);
    for (int j = 1; j < 2000; ++j) {
        const double t = j * tau;
        const double term = exp(lognorm - x * cosh(t) + nu * t) * 0.5 * (1. + exp(-2. * nu * t));
        sum += term;
        if (term < 1e-18 * sum && x * cosh(t) > nu * t + 50.) break;
    }
    return sum * tau;
}

}  // namespace gsb
