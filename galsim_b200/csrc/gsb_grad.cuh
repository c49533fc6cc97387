// Analytic derivatives of the leaf Fourier transforms, for the adjoint of the drawing path.
//
// Every leaf value is v = flux * phi(k') with k' = (kxp, kyp) = (A kx + C ky, B kx + D ky)
// (SBProfile::drawK, src/SBProfile.cpp:400-424).  leaf_grad returns v together with
//   unit = dv/dflux,   gx = dv/dkxp,   gy = dv/dkyp,   gn = dv/dn (Sersic, at fixed r0),
// from which the adjoint forms dv/dA = gx kx, dv/dB = gy kx, dv/dC = gx ky, dv/dD = gy ky.
// The size parameters need no separate derivative: every radial leaf depends on its size s and
// its Jacobian only through s * J, so d/d(ln s) = sum_ij J_ij d/dJ_ij (and per axis for Box).
// Clipped points (Gaussian / Exponential fill rules) have zero derivative, as the clip masks
// are piecewise constant in the parameters.
#pragma once

#include "gsb_profiles.cuh"

namespace gsb {

template <typename T>
struct LeafD { T v, unit, gx, gy, gn; };

// d/dx sinc(x), sinc(x) = sin(pi x) / (pi x):  (cos(pi x) - sinc(x)) / x, series near 0.
template <typename T>
__device__ inline T dsinc_ref(T x)
{
    if (fabs(x) < T(1e-4)) return T(-kPi * kPi / 3.) * x;
    return (cospi(x) - sinpi(x) / (T(kPi) * x)) / x;
}

// Sersic phi(u) = f(ln sqrt(u) - front) / u from the spline (as sersic_kvalue), with
// dphi/du and dphi/dn: the spline of the node derivatives (total derivatives along the moving
// nodes) minus the shift of the spline argument with front(n).
template <typename T>
__device__ inline void sersic_phi_grad(const SersicTableView& tb, const SersicDnView& dn, T u,
                                       T& phi, T& dphidu, T& dphidn)
{
    if (u >= T(tb.ksq_max)) {
        const T a = T(tb.highk_a), b = T(tb.highk_b);
        const T isq = T(1) / sqrt(u), iu = T(1) / u;
        phi = (a + b * isq) * iu;
        dphidu = -(a + T(1.5) * b * isq) * iu * iu;
        dphidn = (T(dn.dhigha) + T(dn.dhighb) * isq) * iu;
        return;
    }
    if (u < T(tb.ksq_min)) {
        const T k2 = T(tb.kderiv2), k4 = T(tb.kderiv4);
        phi = T(1) + u * (k2 + u * k4);
        dphidu = k2 + T(2) * u * k4;
        dphidn = u * (T(dn.dkd2) + u * T(dn.dkd4));
        return;
    }
    const T lk = T(0.5) * log(u) - T(tb.front);
    int i = int(ceil(lk / T(tb.da)));
    if (i >= tb.n) i = tb.n - 1;
    if (i <= 0) i = 1;
    const double4 n0 = tb.node[i - 1], n1 = tb.node[i];
    const T h = T(tb.da);
    const T aa = T(0.5) * log(T(n1.w) / u);      // as in the forward lookup
    const T bb = h - aa;
    const T Q = (aa + h) * T(n0.z) + (bb + h) * T(n1.z);
    const T P = aa * bb;
    const T f = (aa * T(n0.y) + bb * T(n1.y) - (T(1) / T(6)) * P * Q) / h;
    const T fl = ((T(n1.y) - T(n0.y)) - (T(1) / T(6)) * ((aa - bb) * Q + P * (T(n1.z) - T(n0.z)))) / h;
    const double4 d0 = dn.node[i - 1], d1 = dn.node[i];
    const T Qn = (aa + h) * T(d0.z) + (bb + h) * T(d1.z);
    const T fn = (aa * T(d0.y) + bb * T(d1.y) - (T(1) / T(6)) * P * Qn) / h;
    const T iu = T(1) / u;
    phi = f * iu;
    dphidu = (T(0.5) * fl - f) * iu * iu;
    // the argument lk = ln k - front(n) moves with the grid origin
    dphidn = (fn - T(dn.dfront) * fl) * iu;
}

// Moffat: K(x) = c_nu x^nu K_nu(x) and K'(x) / x = -c_nu x^(nu-1) K_(nu-1)(x)
// (DLMF 10.29.4: d/dx [x^nu K_nu(x)] = -x^nu K_(nu-1)(x)), by the same trapezoid rule as
// moffat_kv on K_(nu-1)(x) = int_0^inf exp(-x cosh t) cosh((nu-1) t) dt.
template <typename T>
__device__ inline T moffat_dkv_over_x(T nu, T lognorm_nu, T x)
{
    if (x <= T(0)) return T(0);
    const T tau = sizeof(T) == 4 ? T(0.25) : T(0.125);
    const T m = nu - T(1);
    const T ln = lognorm_nu + m * log(x);
    T sum = T(0.5) * exp(ln - x);
    const int jmax = sizeof(T) == 4 ? 100 : 400;
    for (int j = 1; j < jmax; ++j) {
        const T t = j * tau;
        const T e0 = ln - x * cosh(t);
        const T term = T(0.5) * (exp(e0 + m * t) + exp(e0 - m * t));
        sum += term;
        if (e0 + fabs(m) * t < T(-45)) break;
    }
    return -sum * tau;
}

// d/dt of airy_kvalue: the overlap area of two discs of radii r, s at centre distance d
// changes as dA/dd = -(length of the common chord), so dA/dt = -h / d with h the half chord
// (t = d^2, zero where the discs are disjoint or nested).
template <typename T>
__device__ inline T airy_half_chord_same(T rsq, T t)
{
    if (t >= T(4) * rsq) return T(0);
    return sqrt(fmax(rsq - t / T(4), T(0)));
}

template <typename T>
__device__ inline T airy_half_chord_two(T r, T s, T rsq, T ssq, T t)
{
    const T rps_sq = (r + s) * (r + s);
    const T rms_sq = (r - s) * (r - s);
    if (t >= rps_sq || t <= rms_sq) return T(0);
    return sqrt(fmax(T(0.5) * (rsq + ssq) - (t * t + rps_sq * rms_sq) / (T(4) * t), T(0)));
}

template <typename T>
__device__ inline T airy_dkvalue_dt(T t, T obs, T obssq)
{
    if (t <= T(0)) return T(0);
    const T d = sqrt(t);
    if (obs == T(0)) return -airy_half_chord_same<T>(T(1), t) / d;
    return (-airy_half_chord_same<T>(T(1), t) + T(2) * airy_half_chord_two<T>(T(1), obs, T(1), obssq, t) -
            airy_half_chord_same<T>(obssq, t)) / d;
}

template <typename T>
__device__ inline LeafD<T> leaf_grad(const LeafParams& L, const SersicTableView* tables,
                                     const SersicDnView* dtables, T kx, T ky, const GridRef& g,
                                     int gi, int gj)
{
    const T A = T(L.jac[0]), B = T(L.jac[1]), C = T(L.jac[2]), D = T(L.jac[3]);
    const T kxp = A * kx + C * ky;
    const T kyp = B * kx + D * ky;
    const T flux = T(L.flux);
    const T q = kxp * kxp + kyp * kyp;
    LeafD<T> r{T(0), T(0), T(0), T(0), T(0)};
    T dq = T(0);   // dv/dq, q = |k'|^2
    switch (L.type) {
      case GSB_GAUSSIAN: {
        const T s = T(L.d[0]);
        const T u = q * s * s;
        T phi, dphi;
        if (!(L.flags & GSB_LEAF_JAC_GENERAL)) {
            const T ax = kxp * s, ay = kyp * s;
            phi = exp(T(-0.5) * ax * ax) * exp(T(-0.5) * ay * ay);
            dphi = T(-0.5) * phi;
        } else {
            if (u > T(L.d[1])) return r;
            if (u < T(L.d[2])) { phi = T(1) - T(0.5) * u * (T(1) - T(0.25) * u); dphi = T(-0.5) + T(0.25) * u; }
            else { phi = exp(T(-0.5) * u); dphi = T(-0.5) * phi; }
        }
        r.unit = phi;
        dq = flux * dphi * s * s;
        break;
      }
      case GSB_EXPONENTIAL: {
        if (!exponential_keep(L, g.dk, g.x0, g.y0, g.m, g.n, gi, gj)) return r;
        const T r0 = T(L.d[0]);
        const T p = T(1) + q * r0 * r0;
        const T phi = T(1) / (p * sqrt(p));
        r.unit = phi;
        dq = flux * T(-1.5) * phi / p * r0 * r0;
        break;
      }
      case GSB_SERSIC: {
        const T r0 = T(L.d[0]);
        T phi, dphi, dphidn;
        sersic_phi_grad<T>(tables[L.table], dtables[L.table], q * r0 * r0, phi, dphi, dphidn);
        r.unit = phi;
        r.gn = flux * dphidn;
        dq = flux * dphi * r0 * r0;
        break;
      }
      case GSB_MOFFAT: {
        const T rD = T(L.d[0]);
        const T k = sqrt(q) * rD;
        const int mode = int(L.d[2]);
        const T knorm = T(L.d[1]);
        T K, dKx;   // K(k) and K'(k) / k
        const T e = exp(-k);
        if (mode == 4) {
            // truncated: the spline in k^2, K'(k) / k = 2 dK / d(k^2) (the table held fixed)
            const double4* nd = reinterpret_cast<const double4*>(__double_as_longlong(L.d[6]));
            T dv;
            K = moffat_trunc_kvalue<T>(nd, int(L.d[5]), T(L.d[3]), T(L.d[4]), q * rD * rD, &dv);
            dKx = T(2) * dv;
        } else if (mode == 1) { K = e; dKx = k > T(0) ? -e / k : T(0); }
        else if (mode == 2) { K = e * (T(1) + k); dKx = -e; }
        else if (mode == 3) { K = e * (T(3) + (T(3) + k) * k) * T(1. / 3.); dKx = -e * (T(1) + k) * T(1. / 3.); }
        else { K = moffat_kv<T>(T(L.d[3]), T(L.d[4]), k); dKx = moffat_dkv_over_x<T>(T(L.d[3]), T(L.d[4]), k); }
        r.v = knorm * K;
        r.unit = K;
        dq = knorm * dKx * rD * rD * T(0.5);
        r.gx = T(2) * dq * kxp;
        r.gy = T(2) * dq * kyp;
        return r;
      }
      case GSB_KOLMOGOROV: {
        const T ik0 = T(L.d[0]);
        const T u = q * ik0 * ik0;
        const T u56 = kolm_pow56<T>(u);
        const T phi = exp(-u56);
        r.unit = phi;
        dq = u > T(0) ? flux * T(-5. / 6.) * u56 / u * phi * ik0 * ik0 : T(0);
        break;
      }
      case GSB_AIRY: {
        const T s = T(L.d[0]);
        const T obs = T(L.d[2]), obssq = T(L.d[3]);
        const T t = q * s * s;
        const T unorm = T(1) / (T(kPi) * (T(1) - obssq));   // knorm / flux
        const T a = airy_kvalue<T>(t, obs, obssq);
        r.v = T(L.d[1]) * a;
        r.unit = unorm * a;
        dq = T(L.d[1]) * airy_dkvalue_dt<T>(t, obs, obssq) * s * s;
        r.gx = T(2) * dq * kxp;
        r.gy = T(2) * dq * kyp;
        return r;
      }
      case GSB_BOX: {
        const T wx = T(L.d[0]), wy = T(L.d[1]);
        const T sx = sinc_ref<T>(kxp * wx), sy = sinc_ref<T>(kyp * wy);
        r.unit = sx * sy;
        r.v = flux * r.unit;
        r.gx = flux * wx * dsinc_ref<T>(kxp * wx) * sy;
        r.gy = flux * wy * sx * dsinc_ref<T>(kyp * wy);
        return r;
      }
    }
    r.v = flux * r.unit;
    r.gx = T(2) * dq * kxp;
    r.gy = T(2) * dq * kyp;
    return r;
}

}  // namespace gsb
