// Leaf profile Fourier transforms, evaluated per k-point on the device.
//
// A leaf is drawn at image-space wave vector (kx, ky) through its composed Jacobian
// [A, B, C, D]:  kx' = A kx + C ky,  ky' = B kx + D ky   (SBProfile::drawK,
// src/SBProfile.cpp:400-424).  The reference fills whole k-images with per-profile loops
// whose clipping rules differ between the "1-d" fill (diagonal Jacobian, quadrant
// mirroring) and the "2-d" fill (general Jacobian); both are reproduced here per point.
#pragma once

#include "gsb_internal.cuh"

namespace gsb {

// ---------------------------------------------------------------------------------------
// Exponential clipping ranges (FP64, as in the reference).
// GetKValueRange1d / GetKValueRange2d: src/SBProfile.cpp:508-588.  Keep column i of a row
// iff i1 <= i < i2.  The 2-d test deliberately keeps the reference's `ky0 + m + dky`.
// ---------------------------------------------------------------------------------------
__device__ inline void kvalue_range_1d(int m, double kmax, double ksqmax, double kx0, double dkx,
                                       double ky, int& i1, int& i2)
{
    if (fabs(ky) >= kmax) { i1 = i2 = m; return; }
    const double kysq = ky * ky;
    const double dsq = ksqmax - kysq;
    const double kend = kx0 + m * dkx;
    if (kx0 * kx0 > dsq || kend * kend > dsq) {
        const double d = sqrt(dsq);
        double a = ceil((-kx0 - d) / dkx), b = floor((-kx0 + d) / dkx);
        if (a > b) { const double t = a; a = b; b = t; }
        b += 1.;
        if (b <= 0. || a >= m) { i1 = i2 = m; return; }
        i1 = a < 0. ? 0 : int(a);
        i2 = b > m ? m : int(b);
    } else { i1 = 0; i2 = m; }
}

__device__ inline void kvalue_range_2d(int m, double kmax, double ksqmax, double kx0, double dkx,
                                       double ky0, double dky, int& i1, int& i2)
{
    if (fabs(kx0) > kmax || fabs(kx0 + m * dkx) > kmax || fabs(ky0) > kmax ||
        fabs(ky0 + m + dky) > kmax) {
        const double a = dkx * dkx + dky * dky;
        const double b = dkx * kx0 + dky * ky0;
        const double c = kx0 * kx0 + ky0 * ky0 - ksqmax;
        double d = b * b - a * c;
        if (d <= 0.) { i1 = i2 = m; return; }
        d = sqrt(d);
        double lo = ceil((-b - d) / a), hi = floor((-b + d) / a);
        if (lo > hi) { const double t = lo; lo = hi; hi = t; }
        hi += 1.;
        if (hi <= 0. || lo >= m) { i1 = i2 = m; return; }
        i1 = lo < 0. ? 0 : int(lo);
        i2 = hi > m ? m : int(hi);
    } else { i1 = 0; i2 = m; }
}

// Whether grid point (i, j) (0-based column / row of a k-image whose lower-left corner is at
// integer k index (gx0, gy0), with m columns and n rows) survives the Exponential's clip.
__device__ inline bool exponential_keep(const LeafParams& L, double dk, int gx0, int gy0, int m,
                                        int n, int i, int j)
{
    const double r0 = L.d[0], ksqmax = L.d[1], kmax = L.d[2];
    const double x0 = gx0 * dk, y0 = gy0 * dk;
    if (!(L.flags & GSB_LEAF_JAC_GENERAL)) {
        const double A = L.jac[0], D = L.jac[3];
        const int izero = gx0 < 0 ? -gx0 : 0;
        const int jzero = gy0 < 0 ? -gy0 : 0;
        const double dkx = dk * A * r0, dky = dk * D * r0;
        if (izero != 0 || jzero != 0) {
            // FillQuadrant (src/SBProfile.cpp:434-488): a quadrant image of
            // max(m1,m2)+1 columns is filled from k = (m1==0 ? x0 : 0, n1==0 ? y0 : 0).
            const int m1 = izero, n1 = jzero;
            const int m2 = m - m1 - 1;
            const int mq = (m1 > m2 ? m1 : m2) + 1;
            const double qx0 = (m1 == 0 ? x0 * A : 0.) * r0;
            const double qy0 = (n1 == 0 ? y0 * D : 0.) * r0;
            const int iq = i - m1 < 0 ? m1 - i : i - m1;
            const int jq = j - n1 < 0 ? n1 - j : j - n1;
            int i1, i2;
            kvalue_range_1d(mq, kmax, ksqmax, qx0, dkx, qy0 + jq * dky, i1, i2);
            return iq >= i1 && iq < i2;
        } else {
            int i1, i2;
            kvalue_range_1d(m, kmax, ksqmax, x0 * A * r0, dkx, (y0 * D + j * dk * D) * r0, i1, i2);
            return i >= i1 && i < i2;
        }
    } else {
        const double A = L.jac[0], B = L.jac[1], C = L.jac[2], D = L.jac[3];
        const double kx0 = (A * x0 + C * y0) * r0 + j * (C * dk * r0);
        const double ky0 = (B * x0 + D * y0) * r0 + j * (D * dk * r0);
        int i1, i2;
        kvalue_range_2d(m, kmax, ksqmax, kx0, A * dk * r0, ky0, B * dk * r0, i1, i2);
        return i >= i1 && i < i2;
    }
}

// ---------------------------------------------------------------------------------------
// Sersic FT spline lookup (SersicInfo::kValue, src/SBSersic.cpp:363-376; TSpline::_interp,
// src/Table.cpp:571-586 with ArgVec::upperIndex equal-spacing branch, :73-85).  The node's .w
// holds its k^2.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ inline T sersic_kvalue(const SersicTableView& tb, T ksq)
{
    if (ksq >= T(tb.ksq_max)) {
        return (T(tb.highk_a) + T(tb.highk_b) / sqrt(ksq)) / ksq;
    } else if (ksq < T(tb.ksq_min)) {
        return T(1) + ksq * (T(tb.kderiv2) + ksq * T(tb.kderiv4));
    } else {
        const T lk = T(0.5) * log(ksq) - T(tb.front);
        int i = int(ceil(lk / T(tb.da)));
        if (i >= tb.n) i = tb.n - 1;
        if (i <= 0) i = 1;
        const double4 n0 = tb.node[i - 1];
        const double4 n1 = tb.node[i];
        // the offset from the upper node as the log of a ratio near 1 (accurate in FP32, unlike
        // the difference of two logarithms of size ~10); the spacing is the table's own
        const T h = T(tb.da);
        const T aa = T(0.5) * log(T(n1.w) / ksq);
        const T bb = h - aa;
        const T f = (aa * T(n0.y) + bb * T(n1.y) -
                     (T(1) / T(6)) * aa * bb * ((aa + h) * T(n0.z) + (bb + h) * T(n1.z))) / h;
        return f / ksq;
    }
}

// Truncated Moffat FT at ksq = (k rD)^2 (kV_trunc, src/SBMoffat.cpp:339-345): 0 beyond the
// table's last argument, else its natural cubic spline in k^2 (TSpline, src/Table.cpp:553-686)
// over nodes (k_i^2, v_i, y2_i), k_i = i dk up to rounding of the running sum.  The interval is
// the one the reference's lookup finds (k_{i-1}^2 <= ksq <= k_i^2): first guessed from
// sqrt(ksq) / dk, then moved to the node that brackets ksq.  The offsets from the nodes are
// taken in k (x_i - ksq = (k_i - k)(k_i + k)), which keeps their FP32 rounding relative to
// k rather than to k^2.  *dv (when given) receives the spline's derivative d v / d ksq.
template <typename T>
__device__ inline T moffat_trunc_kvalue(const double4* nd, int n, T dk, T ksq_max, T ksq, T* dv = nullptr)
{
    if (ksq > ksq_max) { if (dv) *dv = T(0); return T(0); }
    const T k = sqrt(ksq);
    int i = int(ceil(k / dk));
    if (i > n - 1) i = n - 1;
    if (i < 1) i = 1;
    for (int it = 0; it < 2 && i < n - 1 && ksq > T(nd[i].x); ++it) ++i;
    for (int it = 0; it < 2 && i > 1 && ksq < T(nd[i - 1].x); ++it) --i;
    const double4 n0 = nd[i - 1];
    const double4 n1 = nd[i];
    const T h = T(n1.x - n0.x);
    const T k0 = T(sqrt(n0.x)), k1 = T(sqrt(n1.x));
    const T aa = (k1 - k) * (k1 + k) / h;      // (x_i - ksq) / h
    const T bb = (k - k0) * (k + k0) / h;      // (ksq - x_{i-1}) / h
    const T y0 = T(n0.y), y1 = T(n1.y), z0 = T(n0.z), z1 = T(n1.z);
    if (dv) *dv = (y1 - y0) / h + (-(T(3) * aa * aa - T(1)) * z0 + (T(3) * bb * bb - T(1)) * z1) * h * T(1. / 6.);
    return aa * y0 + bb * y1 + ((aa * aa * aa - aa) * z0 + (bb * bb * bb - bb) * z1) * (h * h) * T(1. / 6.);
}

// c_nu x^nu K_nu(x) normalised to 1 at x = 0, by the trapezoid rule on
// K_nu(x) = int_0^inf exp(-x cosh t) cosh(nu t) dt (DLMF 10.32.9).
template <typename T>
__device__ inline T moffat_kv(T nu, T lognorm_nu, T x)
{
    if (x <= T(0)) return T(1);
    const T tau = sizeof(T) == 4 ? T(0.25) : T(0.125);
    const T ln = lognorm_nu + nu * log(x);
    T sum = T(0.5) * exp(ln - x);
    const int jmax = sizeof(T) == 4 ? 100 : 400;
    for (int j = 1; j < jmax; ++j) {
        const T t = j * tau;
        const T ex = ln - x * cosh(t) + nu * t;
        const T term = exp(ex) * T(0.5) * (T(1) + exp(T(-2) * nu * t));
        sum += term;
        if (ex < T(-45) && x * cosh(t) > nu * t + T(10)) break;
    }
    return sum * tau;
}

// ksq^(5/6) for the Kolmogorov FT exp(-(k/k0)^(5/3)).  FP32: exp2(5/6 log2 ksq) with the
// hardware log2 (absolute error ~2^-21 in log2), which moves exp(-u) by < 1e-7 of the flux;
// FP64: pow.
template <typename T>
__device__ inline T kolm_pow56(T ksq) { return pow(ksq, T(5. / 6.)); }
template <>
__device__ inline float kolm_pow56<float>(float ksq)
{ return ksq > 0.f ? exp2f(__log2f(ksq) * (5.f / 6.f)) : 0.f; }

template <typename T>
__device__ inline T sinc_ref(T x)
{
    // math::sinc (src/math/Sinc.cpp:29-33): sin(pi x)/(pi x), series below 1e-4.
    if (fabs(x) < T(1e-4)) return T(1) - T(kPi * kPi / 6.) * x * x;
    return sinpi(x) / (T(kPi) * x);
}

// ---------------------------------------------------------------------------------------
// One leaf at image-space (kx, ky).  (gi, gj, ...) locate the point on the reference's
// k-image grid for the Exponential clip.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ inline T leaf_kvalue(const LeafParams& L, const SersicTableView* tables, T kx, T ky,
                                const GridRef& g, int gi, int gj)
{
    const T A = T(L.jac[0]), B = T(L.jac[1]), C = T(L.jac[2]), D = T(L.jac[3]);
    const T kxp = A * kx + C * ky;
    const T kyp = B * kx + D * ky;
    const T flux = T(L.flux);
    switch (L.type) {
      case GSB_GAUSSIAN: {
        const T s = T(L.d[0]);
        if (!(L.flags & GSB_LEAF_JAC_GENERAL)) {
            // separable 1-d fill (SBGaussian.cpp:151-192): no clip, exp per axis
            const T ax = kxp * s, ay = kyp * s;
            return flux * exp(T(-0.5) * ax * ax) * exp(T(-0.5) * ay * ay);
        }
        const T ksq = (kxp * kxp + kyp * kyp) * s * s;
        if (ksq > T(L.d[1])) return T(0);
        if (ksq < T(L.d[2])) return flux * (T(1) - T(0.5) * ksq * (T(1) - T(0.25) * ksq));
        return flux * exp(T(-0.5) * ksq);
      }
      case GSB_EXPONENTIAL: {
        if (!exponential_keep(L, g.dk, g.x0, g.y0, g.m, g.n, gi, gj)) return T(0);
        const T r0 = T(L.d[0]);
        const T ksqp1 = T(1) + (kxp * kxp + kyp * kyp) * r0 * r0;
        return flux / (ksqp1 * sqrt(ksqp1));
      }
      case GSB_SERSIC: {
        const T r0 = T(L.d[0]);
        const T ksq = (kxp * kxp + kyp * kyp) * r0 * r0;
        return flux * sersic_kvalue<T>(tables[L.table], ksq);
      }
      case GSB_MOFFAT: {
        const T rD = T(L.d[0]);
        const int mode = int(L.d[2]);
        const T knorm = T(L.d[1]);
        if (mode == 4) {
            const double4* nd = reinterpret_cast<const double4*>(__double_as_longlong(L.d[6]));
            return knorm * moffat_trunc_kvalue<T>(nd, int(L.d[5]), T(L.d[3]), T(L.d[4]),
                                                  (kxp * kxp + kyp * kyp) * rD * rD);
        }
        const T k = sqrt(kxp * kxp + kyp * kyp) * rD;
        if (mode == 1) return knorm * exp(-k);
        if (mode == 2) return knorm * exp(-k) * (T(1) + k);
        if (mode == 3) return knorm * exp(-k) * (T(3) + (T(3) + k) * k) * T(1. / 3.);
        return knorm * moffat_kv<T>(T(L.d[3]), T(L.d[4]), k);
      }
      case GSB_KOLMOGOROV: {
        const T ik0 = T(L.d[0]);
        const T ksq = (kxp * kxp + kyp * kyp) * ik0 * ik0;
        return flux * exp(-kolm_pow56<T>(ksq));
      }
      case GSB_AIRY: {
        const T s = T(L.d[0]);       // 1 / (D pi)
        const T knorm = T(L.d[1]);
        const T obs = T(L.d[2]), obssq = T(L.d[3]);
        const T t = (kxp * kxp + kyp * kyp) * s * s;   // ksq / (pi D)^2
        return knorm * airy_kvalue<T>(t, obs, obssq);
      }
      case GSB_BOX: {
        return flux * sinc_ref<T>(kxp * T(L.d[0])) * sinc_ref<T>(kyp * T(L.d[1]));
      }
    }
    return T(0);
}

}  // namespace gsb
