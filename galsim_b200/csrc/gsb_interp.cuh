// InterpolatedImage k-values on the device.
//
// An InterpolatedImage leaf is the k interpolant applied to the DFT samples K(p, q) of the
// zero-padded image, times the x interpolant's Fourier transform:
//   v(kx, ky) = flux * U(kx / 2 pi) U(ky / 2 pi) * sum_pq w(p - kx N / 2 pi) w(q - ky N / 2 pi) K(p, q)
// (SBInterpolatedImage::kValue and both fillKImage forms, src/SBInterpolatedImage.cpp:385-448,
// 767-1000), with K periodic in N and Hermitian (K(-p, -q) = conj K(p, q)), so only the half
// plane p = 0..N/2 is stored (p-major: N/2 + 1 columns of N values q).  Tap positions are formed in
// FP64 even for FP32 draws: their fractions must stay exact at indices of several hundred.
#pragma once

#include "gsb_fft.cuh"
#include "gsb_profiles.cuh"

namespace gsb {

// Real-space kernels (src/Interpolant.cpp:171-176 Nearest, 245-249 Linear, 284-290 Cubic,
// 389-432 Quintic; the quintic of Bernstein & Gruen 2014, arXiv:1401.2636, in its form with
// vanishing fourth derivative of the step response).
template <typename T>
__device__ __forceinline__ T interp_xval(int code, T x)
{
    x = fabs(x);
    switch (code) {
      case GSB_INTERP_NEAREST:
        return x > T(0.5) ? T(0) : T(1);
      case GSB_INTERP_LINEAR:
        return x > T(1) ? T(0) : T(1) - x;
      case GSB_INTERP_CUBIC:
        if (x < T(1)) return T(1) + x * x * (T(1.5) * x - T(2.5));
        if (x < T(2)) return T(-0.5) * (x - T(1)) * (x - T(2)) * (x - T(2));
        return T(0);
      case GSB_INTERP_QUINTIC:
        if (x <= T(1)) return T(1) + x * x * x * (T(-95. / 12.) + x * (T(23. / 2.) + x * T(-55. / 12.)));
        if (x <= T(2))
            return (x - T(1)) * (x - T(2)) *
                   (T(-23. / 4.) + x * (T(29. / 2.) + x * (T(-83. / 8.) + x * T(55. / 24.))));
        if (x <= T(3))
            return (x - T(2)) * (x - T(3)) * (x - T(3)) * (T(-9. / 4.) + x * (T(25. / 12.) + x * T(-11. / 24.)));
        return T(0);
    }
    return T(0);
}

// Half-width of the kernel support in samples (Interpolant::xrange, include/galsim/Interpolant.h).
__host__ __device__ inline double interp_xrange(int code)
{
    switch (code) {
      case GSB_INTERP_NEAREST: return 0.5;
      case GSB_INTERP_LINEAR: return 1.;
      case GSB_INTERP_CUBIC: return 2.;
      case GSB_INTERP_QUINTIC: return 3.;
    }
    return 0.;
}

// Fourier transforms of the kernels, u in cycles per sample (the closed forms of
// src/Interpolant.cpp:176, 251-255, 292-302, 435-461, derived from the piecewise polynomials).
template <typename T>
__device__ __forceinline__ T interp_uval(int code, T u)
{
    if (code == GSB_INTERP_DELTA) return T(1);
    if (code == GSB_INTERP_SINC) {
        const T a = fabs(u);
        return a > T(0.5) ? T(0) : (a < T(0.5) ? T(1) : T(0.5));
    }
    const T s = sinc_ref<T>(u);
    switch (code) {
      case GSB_INTERP_NEAREST: return s;
      case GSB_INTERP_LINEAR: return s * s;
      case GSB_INTERP_CUBIC: {
        const T c = cospi(u);
        return s * s * s * (T(3) * s - T(2) * c);
      }
      case GSB_INTERP_QUINTIC: {
        const T c = cospi(u);
        const T ssq = s * s;
        const T piusq = T(kPi * kPi) * u * u;
        return s * ssq * ssq * (s * (T(55) - T(19) * piusq) + T(2) * c * (piusq - T(27)));
      }
    }
    return T(0);
}

// Extent of the kernel's transform, beyond which |U| < kvalue_accuracy (Interpolant::urange:
// include/galsim/Interpolant.h:237, 278, 347; src/Interpolant.cpp:364-368, 518-523).
__host__ __device__ inline double interp_urange(int code, double kacc)
{
    switch (code) {
      case GSB_INTERP_DELTA: return 1. / kacc;
      case GSB_INTERP_NEAREST: return 1. / (kPi * kacc);
      case GSB_INTERP_LINEAR: return sqrt(1. / kacc) / kPi;
      case GSB_INTERP_CUBIC: return pow((3. * sqrt(3.) / 8.) / kacc, 1. / 3.) / kPi;
      case GSB_INTERP_QUINTIC: return pow((25. * sqrt(5.) / 108.) / kacc, 1. / 3.) / kPi;
      case GSB_INTERP_SINC: return 0.5;
    }
    return 0.;
}

// The Lanczos transform from its table (Lanczos::uval, src/Interpolant.cpp:914-919): 0 above
// uMax, else the natural cubic spline through the nodes, found as the reference's Table finds
// an interval of equally spaced arguments (the first node index i >= 1 with u <= u_i,
// i = ceil((u - u_0) / du) clipped to 1..n-1).  Table layout: header {n, du, u_0, uMax}, then
// {u, F, F'', 0} per node.
__device__ inline double table_uval(const double* tab, double u)
{
    u = fabs(u);
    const double4 hd = reinterpret_cast<const double4*>(tab)[0];
    if (u > hd.w) return 0.;
    const int n = int(hd.x);
    const double4* nd = reinterpret_cast<const double4*>(tab) + 1;
    double fi = ceil((u - hd.z) / hd.y);
    int i = fi < 1. ? 1 : (fi > double(n - 1) ? n - 1 : int(fi));
    const double4 a = nd[i - 1], b = nd[i];
    const double h = b.x - a.x;
    const double aa = (b.x - u) / h;
    const double bb = 1. - aa;
    return aa * a.y + bb * b.y + ((aa * aa * aa - aa) * a.z + (bb * bb * bb - bb) * b.z) * (h * h) / 6.;
}

// The Lanczos kernel as the k interpolant (Lanczos::xCalc, src/Interpolant.cpp:563-716):
// n sin(pi x) sin(pi x / n) / (pi x)^2 for |x| < n (sin(pi x) from sin(pi x / n) by the
// multiple-angle identities for n = 2, 3; the two-term series below |x| = 1e-4), divided, with
// conserve_dc, by the DC-correcting factor 1 - sum_j 2 K_j (1 - cos(2 pi j x)), j = 1..5,
// written as the reference writes it in powers of s^2 = sin^2(pi x).  kt = {n, conserve_dc,
// K_1 .. K_5, 0}, K_j the kernel's transform at u = j.
template <typename T>
__device__ __forceinline__ T lanczos_xval(const double* kt, T x)
{
    x = fabs(x);
    const int n = int(kt[0]);
    const T nd = T(n);
    if (x >= nd) return T(0);
    constexpr T kPiT = T(3.141592653589793238462643383279502884);
    T res, s;
    if (x > T(1.e-4)) {
        if (n == 1) {
            s = sinpi(x);
            const T t = s / (kPiT * x);
            res = t * t;
        } else if (n == 2) {
            T sn, cn;
            sincospi(x / T(2), &sn, &cn);
            s = T(2) * sn * cn;
            res = (T(2) / (kPiT * kPiT)) * s * sn / (x * x);
        } else if (n == 3) {
            const T sn = sinpi(x / T(3));
            s = sn * (T(3) - T(4) * sn * sn);
            res = (T(3) / (kPiT * kPiT)) * s * sn / (x * x);
        } else {
            s = sinpi(x);
            const T sn = sinpi(x / nd);
            res = (nd / (kPiT * kPiT)) * s * sn / (x * x);
        }
    } else {
        const T pix = kPiT * x;
        const T t = (T(1) / T(6)) * pix * pix;
        s = pix * (T(1) - t);
        res = T(1) - t * (T(1) + T(1) / (nd * nd));
    }
    if (kt[1] != 0.) {
        const T q = s * s;
        const T K1 = T(kt[2]), K2 = T(kt[3]), K3 = T(kt[4]), K4 = T(kt[5]), K5 = T(kt[6]);
        const T f = T(1) - T(4) * K1 * q - T(16) * K2 * q * (T(1) - q) -
                    T(4) * K3 * q * (T(9) - q * (T(24) - T(16) * q)) -
                    T(64) * K4 * q * (T(1) - q * (T(5) - q * (T(8) - T(4) * q))) -
                    T(4) * K5 * q * (T(25) - q * (T(200) - q * (T(560) - q * (T(640) - T(256) * q))));
        res /= f;
    }
    return res;
}

// K(p, q) of the half-plane k-image (stored p-major: K[p N + q], p = 0..N/2) for p, q already
// reduced to 0..N-1.
template <typename T>
__device__ __forceinline__ Cx<T> kimage_at(const Cx<T>* K, int N, int pm, int qm)
{
    if (pm <= N / 2) return K[(size_t)pm * N + qm];
    const Cx<T> v = K[(size_t)(N - pm) * N + (qm == 0 ? 0 : N - qm)];
    return cx<T>(v.x, -v.y);
}

constexpr int kInterpMaxTaps = 8;   // 2 xrange + 1 for the widest kernel (quintic: 7)

// The taps of one axis at one k: first sample index (already reduced mod N), count, and the
// kernel weights w[t] = xval(p1 + t - s), with the x interpolant's transform (and, for the
// x axis, the leaf flux) folded in.
template <typename T>
struct IITaps {
    int p0;
    int n;
    T w[kInterpMaxTaps];
};

// Taps of the axis with k' = kp: s = kp N / 2 pi.  `shortcut`: the separable fill's single tap
// at (near-)integer positions (SBInterpolatedImage.cpp:829-834).  Outside the x interpolant's
// support (|k'| > maxk1, SBInterpolatedImage.cpp:394 and 786-789) there are no taps.  The
// transform factor is evaluated in FP64 for every precision: the quintic's
// s (55 - 19 pi^2 u^2) + 2 c (pi^2 u^2 - 27) is 55 s - 54 c + O(u^2) near u = 0, which would
// amplify FP32 rounding of s and c 55-fold (a 3e-6 flux bias).
template <typename T>
__device__ __noinline__ void ii_axis_taps(const LeafParams& L, double kp, bool shortcut, bool with_flux,
                                             IITaps<T>& e)
{
    e.n = 0;
    e.p0 = 0;
    if (fabs(kp) > L.d[1]) return;
    const int N = int(L.d[4]);
    const int codes = int(L.d[2]);
    const int xc = codes & 15, kc = codes >> 4;
    const double* kt = reinterpret_cast<const double*>(__double_as_longlong(L.d[3]));
    const double s = kp * L.d[0];
    constexpr double kSmall = 10. * 2.220446049250313e-16;
    const double fl = floor(s + 0.01);
    int p1, p2;
    if (shortcut && fabs(s - fl) < kSmall * (fabs(s) + 1.)) {
        p1 = p2 = int(fl);
    } else {
        const double xr = kc == GSB_INTERP_LANCZOS ? kt[0] : interp_xrange(kc);
        p1 = int(ceil(s - xr));
        p2 = int(floor(s + xr));
    }
    int n = p2 - p1 + 1;
    n = n < 0 ? 0 : (n > kInterpMaxTaps ? kInterpMaxTaps : n);
    constexpr double kUscale = 1. / (2. * kPi);
    const double ux = kp * kUscale;
    const double u = (xc == GSB_INTERP_LANCZOS
                          ? table_uval(reinterpret_cast<const double*>(__double_as_longlong(L.d[5])), ux)
                          : interp_uval<double>(xc, ux)) * (with_flux ? L.flux : 1.);
    // p - s = (p - p1) + (p1 - s): an integer plus a fraction, exact before the rounding to T
    const T off = T(double(p1) - s);
#pragma unroll
    for (int t = 0; t < kInterpMaxTaps; ++t)
        e.w[t] = t < n ? T(u * double(kc == GSB_INTERP_LANCZOS ? lanczos_xval<T>(kt, T(t) + off)
                                                              : interp_xval<T>(kc, T(t) + off)))
                       : T(0);
    int pw = p1 % N;
    e.p0 = pw < 0 ? pw + N : pw;
    e.n = n;
}

// sum_ab wy_b wx_a K(p0x + a, p0y + b) over the taps of both axes.
template <typename T>
__device__ __noinline__ Cx<T> ii_sum(const LeafParams& L, const IITaps<T>& ex, const IITaps<T>& ey)
{
    const int N = int(L.d[4]);
    const Cx<T>* K = reinterpret_cast<const Cx<T>*>(
        __double_as_longlong(sizeof(T) == 8 ? L.d[6] : L.d[7]));
    Cx<T> sum = cx<T>(T(0), T(0));
    int qw = ey.p0;
    for (int b = 0; b < ey.n; ++b) {
        const T wy = ey.w[b];
        if (wy != T(0)) {
            Cx<T> row = cx<T>(T(0), T(0));
            int pw = ex.p0;
            for (int a = 0; a < ex.n; ++a) {
                const Cx<T> v = kimage_at<T>(K, N, pw, qw);
                row.x += ex.w[a] * v.x;
                row.y += ex.w[a] * v.y;
                if (++pw == N) pw = 0;
            }
            sum.x += wy * row.x;
            sum.y += wy * row.y;
        }
        if (++qw == N) qw = 0;
    }
    return sum;
}

// InterpolatedImage leaf at k index (i, j) of a grid with spacing dk.
// d[0] = (N/2) / pi (k to sample index), d[1] = maxk1 (x interpolant cut-off), d[2] / d[3] =
// x interpolant code + 16 k interpolant code, d[3] = the k interpolant's coefficient block
// address (Lanczos), d[4] = N, d[5] = the x interpolant's table address (Lanczos), d[6] / d[7] =
// FP64 / FP32 k-image addresses.
template <typename T>
__device__ __noinline__ Cx<T> ii_kvalue(const LeafParams& L, double dk, int i, int j)
{
    const double kx = i * dk, ky = j * dk;
    const double kxp = L.jac[0] * kx + L.jac[2] * ky;
    const double kyp = L.jac[1] * kx + L.jac[3] * ky;
    const double maxk1 = L.d[1];
    if (fabs(kxp) > maxk1 || fabs(kyp) > maxk1) return cx<T>(T(0), T(0));
    const bool sep = !(L.flags & GSB_LEAF_JAC_GENERAL);
    IITaps<T> ex, ey;
    ii_axis_taps<T>(L, kxp, sep, true, ex);
    ii_axis_taps<T>(L, kyp, sep, false, ey);
    return ii_sum<T>(L, ex, ey);
}

}  // namespace gsb
