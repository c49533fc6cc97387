// Real-space drawing (drawReal) of profiles that are analytic in real space: sums and affine
// transformations of Gaussian, Exponential, Sersic, Moffat, Kolmogorov, Airy and Box leaves,
// each leaf given with its composed Jacobian, offset and flux scaling (gsb_xleaf).  One CTA per
// stamp (grid-stride over the stamps): the leaves' pixel-grid mappings and normalisations
// (SBProfile::draw, src/SBProfile.cpp:305-383, and the profiles' constructors) are formed
// once per stamp in shared memory, then the threads sweep the stamp's pixels row-major, each
// summing the leaves' xValues in FP64.  Compute-bound (one transcendental or a spline lookup
// per leaf and pixel); the output write is the only HBM traffic.
#include <algorithm>

#include "gsb_internal.cuh"
#include "gsb_interp.cuh"

namespace gsb {

// KolmogorovInfo's radial spline for these GSParams (gsb_tables.cu).
int kolmogorov_radial(const gsb_gsparams* gsp, cudaStream_t stream, const double4** nodes, int* n);

namespace {

struct XLeafC {
    int type, mode;            // mode: 0 no Jacobian, 1 diagonal, 2 general
    double u0, du, duy;        // u = u0 + i du + j duy   (profile frame)
    double v0, dv, dvx;        // v = v0 + j dv + i dvx
    double amp;                // flux_ratio x the Jacobian's area factor
    double c[6];               // per-type constants
    const double4* node;       // Kolmogorov radial spline
    int nnode;
    // InterpolatedImage: the region, its frame position and size, the x interpolant and its
    // half-width, a Lanczos kernel's coefficients
    const double* region;
    int rx0, ry0, rnx, rny, xc;
    double xr;
    const double* ktab;
};

// SBProfile::draw's pixel-grid mapping for one leaf (imscale 1; x0 = xmin - xoff).
__device__ void setup_grid(XLeafC& C, const gsb_xleaf& L, int xmin, int ymin)
{
    const double x0 = xmin - L.xoff, y0 = ymin - L.yoff;
    double amp = L.flux_ratio;
    if (!(L.flags & GSB_XLEAF_JAC)) {
        C.mode = 0;
        C.u0 = x0; C.du = 1.; C.duy = 0.;
        C.v0 = y0; C.dv = 1.; C.dvx = 0.;
    } else if (L.jac[1] == 0. && L.jac[2] == 0.) {
        C.mode = 1;
        const double xs = 1. / L.jac[0], ys = 1. / L.jac[3];
        C.u0 = x0 * xs; C.du = xs; C.duy = 0.;
        C.v0 = y0 * ys; C.dv = ys; C.dvx = 0.;
        amp *= fabs(xs * ys);
    } else {
        C.mode = 2;
        const double A = L.jac[0], B = L.jac[1], Cc = L.jac[2], D = L.jac[3];
        const double invdet = 1. / (A * D - B * Cc);
        C.u0 = (D * x0 - B * y0) * invdet;
        C.v0 = (-Cc * x0 + A * y0) * invdet;
        C.du = D * invdet; C.duy = -B * invdet;
        C.dv = A * invdet; C.dvx = -Cc * invdet;
        amp *= fabs(invdet);
    }
    C.amp = amp;
}

// The profiles' constants (their C++ constructors).
__device__ void setup_profile(XLeafC& C, const gsb_xleaf& L, const gsb_gsparams& gsp, const double4* kolm,
                              int kolm_n)
{
    C.type = L.type;
    C.node = nullptr;
    C.nnode = 0;
    for (int i = 0; i < 6; ++i) C.c[i] = 0.;
    switch (L.type) {
      case GSB_GAUSSIAN: {        // SBGaussian.cpp:57-69
        const double inv_sigma = 1. / L.p[0];
        const double inv_sigma_sq = inv_sigma * inv_sigma;
        C.c[0] = L.flux * inv_sigma_sq / (2. * kPi);
        C.c[1] = inv_sigma_sq;
        break;
      }
      case GSB_EXPONENTIAL: {     // SBExponential.cpp:67-82
        const double inv_r0 = 1. / L.p[0];
        C.c[0] = (L.flux / (2. * kPi)) * (inv_r0 * inv_r0);
        C.c[1] = inv_r0;
        break;
      }
      case GSB_SERSIC: {          // SBSersic.cpp:71-90, 354-361: xnorm = flux / (2 pi n Gamma(2n) F r0^2)
        const double n = L.p[0], r0 = L.p[1], trunc = L.p[2];
        const double inv_r0 = 1. / r0;
        const double gamma2n = tgamma(2. * n);
        const double t = trunc / r0;
        const double ff = trunc > 0. ? gamma_p(2. * n, pow(t, 1. / n)) : 1.;
        C.c[0] = L.flux * (1. / (2. * kPi * n * gamma2n * ff)) * (inv_r0 * inv_r0);
        C.c[1] = inv_r0 * inv_r0;
        C.c[2] = 1. / (2. * n);
        C.c[3] = trunc > 0. ? t * t : -1.;
        break;
      }
      case GSB_MOFFAT: {          // SBMoffat.cpp:163-203
        const double beta = L.p[0], rD = L.p[1], trunc = L.p[2];
        double maxRrD, ff;
        if (trunc > 0.) {
            maxRrD = trunc / rD;
            ff = 1. - pow(1. + maxRrD * maxRrD, 1. - beta);
        } else {
            ff = 1.;
            maxRrD = sqrt(pow(gsp.xvalue_accuracy, 1. / (1. - beta)) - 1.);
        }
        C.c[0] = L.flux * (beta - 1.) / (kPi * ff * rD * rD);
        C.c[1] = 1. / (rD * rD);
        C.c[2] = maxRrD * maxRrD;
        C.c[3] = beta;
        break;
      }
      case GSB_KOLMOGOROV: {      // SBKolmogorov.cpp:85-92
        const double k0 = 2.992939911888651 / L.p[0];
        C.c[0] = L.flux * k0 * k0;
        C.c[1] = k0;
        C.node = kolm;
        C.nnode = kolm_n;
        break;
      }
      case GSB_AIRY: {            // SBAiry.cpp:66-77; the AiryInfo(No)Obs radial functions
        const double D = 1. / L.p[0], obs = L.p[1];
        C.c[0] = L.flux * D * D;
        C.c[1] = D;
        C.c[2] = obs;
        C.c[3] = obs * obs;
        C.c[4] = sqrt(8. * gsp.xvalue_accuracy);
        C.c[5] = obs == 0. ? kPi : kPi / (1. - obs * obs);
        break;
      }
      case GSB_BOX: {             // SBBox.cpp:55-60
        C.c[0] = L.flux / (L.p[0] * L.p[1]);
        C.c[1] = 0.5 * L.p[0];
        C.c[2] = 0.5 * L.p[1];
        break;
      }
      case GSB_INTERPOLATED: {    // the interpolated pixel values (no normalisation of its own)
        C.c[0] = L.flux;
        C.region = L.region;
        C.rx0 = L.rx0; C.ry0 = L.ry0; C.rnx = L.rnx; C.rny = L.rny;
        C.xc = int(L.p[0]);
        C.ktab = L.ktab;
        C.xr = C.xc == GSB_INTERP_LANCZOS ? L.ktab[0]
             : C.xc == GSB_INTERP_SINC ? 1. / (kPi * gsp.kvalue_accuracy) : interp_xrange(C.xc);
        break;
      }
      default:
        C.type = -1;
    }
}

// KolmogorovInfo::xValue: the natural spline of the radial table, 0 beyond its last node
// (the table lookup finds the node interval holding r, src/Table.cpp:78-130).
__device__ double kolm_radial(const double4* nd, int n, double r)
{
    if (n < 2 || !(r < nd[n - 1].x)) return 0.;
    int lo = 0, hi = n - 1;                // nd[lo].x <= r < nd[hi].x
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (nd[mid].x <= r) lo = mid; else hi = mid;
    }
    const double4 a = nd[hi - 1], b = nd[hi];
    const double h = b.x - a.x;
    const double aa = (b.x - r) / h, bb = 1. - aa;
    return aa * a.y + bb * b.y + ((aa * aa * aa - aa) * a.z + (bb * bb * bb - bb) * b.z) * (h * h) / 6.;
}

__device__ double ii_xvalue(const XLeafC& C, double x, double y);

__device__ double xvalue(const XLeafC& C, double u, double v)
{
    switch (C.type) {
      case GSB_GAUSSIAN:
        return C.c[0] * exp(-0.5 * (u * u + v * v) * C.c[1]);
      case GSB_EXPONENTIAL:
        return C.c[0] * exp(-sqrt(u * u + v * v) * C.c[1]);
      case GSB_SERSIC: {
        const double rsq = (u * u + v * v) * C.c[1];
        if (C.c[3] >= 0. && rsq > C.c[3]) return 0.;
        return C.c[0] * exp(-pow(rsq, C.c[2]));
      }
      case GSB_MOFFAT: {
        const double rsq = (u * u + v * v) * C.c[1];
        if (rsq > C.c[2]) return 0.;
        return C.c[0] * pow(1. + rsq, -C.c[3]);
      }
      case GSB_KOLMOGOROV:
        return C.c[0] * kolm_radial(C.node, C.nnode, sqrt(u * u + v * v) * C.c[1]);
      case GSB_INTERPOLATED:
        return C.c[0] * ii_xvalue(C, u, v);
      case GSB_AIRY: {
        const double nu = sqrt(u * u + v * v) * C.c[1] * kPi;
        double x;
        if (nu < C.c[4]) x = C.c[2] == 0. ? 0.5 : 0.5 * (1. - C.c[3]);
        else if (C.c[2] == 0.) x = j1(nu) / nu;
        else x = (j1(nu) - C.c[2] * j1(C.c[2] * nu)) / nu;
        return C.c[0] * (x * x * C.c[5]);
      }
    }
    return 0.;
}

// The x interpolant's kernel (Interpolant::xval): the polynomial kernels, Lanczos::xCalc, and
// sinc(x) for SincInterpolant.
__device__ double ii_xval(const XLeafC& C, double x)
{
    if (C.xc == GSB_INTERP_LANCZOS) return lanczos_xval<double>(C.ktab, x);
    if (C.xc == GSB_INTERP_SINC) return sinc_ref<double>(x);
    return interp_xval<double>(C.xc, x);
}

// SBInterpolatedImage::xValue (SBInterpolatedImage.cpp:167-215): the taps within the x
// interpolant's half-width of (x, y) (a single tap along an axis where the position is an
// integer to 10 eps), clipped to the nonzero region, summed row by row.
__device__ double ii_xvalue(const XLeafC& C, double x, double y)
{
    constexpr double kSmall = 10. * 2.220446049250313e-16;
    int p1, p2, q1, q2;
    const double fx = floor(x + 0.01), fy = floor(y + 0.01);
    if (fabs(x - fx) < kSmall * (fabs(x) + 1.)) { p1 = p2 = int(fx); }
    else { p1 = int(ceil(x - C.xr)); p2 = int(floor(x + C.xr)); }
    if (fabs(y - fy) < kSmall * (fabs(y) + 1.)) { q1 = q2 = int(fy); }
    else { q1 = int(ceil(y - C.xr)); q2 = int(floor(y + C.xr)); }
    const int bx1 = C.rx0 + C.rnx - 1, by1 = C.ry0 + C.rny - 1;
    if (p2 < C.rx0 || p1 > bx1 || q2 < C.ry0 || q1 > by1) return 0.;
    p1 = max(p1, C.rx0); p2 = min(p2, bx1);
    q1 = max(q1, C.ry0); q2 = min(q2, by1);
    double sum = 0.;
    for (int q = q1; q <= q2; ++q) {
        const double* row = C.region + (size_t)(q - C.ry0) * C.rnx - C.rx0;
        double xsum = 0.;
        for (int p = p1; p <= p2; ++p) xsum += ii_xval(C, p - x) * row[p];
        sum += xsum * ii_xval(C, q - y);
    }
    return sum;
}

// SBBox::fillXImage: the diagonal form fills -w/2 <= x < w/2 on the pixel grid, the general
// form |x| < w/2 along each row (SBBox.cpp:79-150).
__device__ double box_value(const XLeafC& C, int i, int j)
{
    if (C.mode <= 1) {
        const double x0 = C.u0 / C.du, y0 = C.v0 / C.dv;
        const double wo2 = C.c[1] / fabs(C.du), ho2 = C.c[2] / fabs(C.dv);
        const bool in = (i >= ceil(-wo2 - x0)) && (i < ceil(wo2 - x0)) && (j >= ceil(-ho2 - y0)) &&
                        (j < ceil(ho2 - y0));
        return in ? C.c[0] : 0.;
    }
    const double x = C.u0 + i * C.du + j * C.duy, y = C.v0 + j * C.dv + i * C.dvx;
    return (fabs(x) < C.c[1] && fabs(y) < C.c[2]) ? C.c[0] : 0.;
}

template <typename T>
__global__ void __launch_bounds__(256) draw_real_kernel(int L, int S, const gsb_gsparams gsp,
                                                        const gsb_xleaf* __restrict__ leaves,
                                                        const gsb_stamp* __restrict__ stamps, const double4* kolm,
                                                        int kolm_n, T* __restrict__ out, int add, double* flux)
{
    __shared__ XLeafC C[GSB_MAX_LEAVES];
    __shared__ double part[8];
    for (int s = blockIdx.x; s < S; s += gridDim.x) {
        const gsb_stamp g = stamps[s];
        if (threadIdx.x < L) {
            const gsb_xleaf& lf = leaves[(size_t)s * L + threadIdx.x];
            setup_grid(C[threadIdx.x], lf, g.xmin, g.ymin);
            setup_profile(C[threadIdx.x], lf, gsp, kolm, kolm_n);
        }
        __syncthreads();
        double fsum = 0.;
        const long long npix = (long long)g.nx * g.ny;
        for (long long p = threadIdx.x; p < npix; p += blockDim.x) {
            const int i = int(p % g.nx), j = int(p / g.nx);
            double val = 0.;
            for (int l = 0; l < L; ++l) {
                const XLeafC& c = C[l];
                double x;
                if (c.type == GSB_BOX) {
                    x = box_value(c, i, j);
                } else {
                    const double u = c.u0 + i * c.du + j * c.duy;
                    const double v = c.v0 + j * c.dv + i * c.dvx;
                    x = xvalue(c, u, v);
                }
                val += c.amp * x;
            }
            const T tv = T(val);
            T* o = out + g.out_offset + p;
            *o = add ? T(*o + tv) : tv;
            fsum += double(tv);
        }
        for (int o = 16; o > 0; o >>= 1) fsum += __shfl_xor_sync(0xffffffffu, fsum, o);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = fsum;
        __syncthreads();
        if (threadIdx.x == 0 && flux) {
            double t = 0.;
            for (int w = 0; w < int(blockDim.x >> 5); ++w) t += part[w];
            flux[s] = t;
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace gsb

extern "C" int gsb_draw_real(int n_leaves, int n_stamps, const gsb_gsparams* gsp, const gsb_xleaf* d_leaves,
                             const gsb_stamp* d_stamps, void* d_out, int out_dtype, int add_to_image,
                             double* d_added_flux, void* stream)
{
    using namespace gsb;
    if (!gsp) return set_error(GSB_ERR_INVALID, "null gsparams");
    if (n_leaves < 1 || n_leaves > GSB_MAX_LEAVES) return set_error(GSB_ERR_INVALID, "n_leaves out of range");
    if (n_stamps < 0) return set_error(GSB_ERR_INVALID, "negative stamp count");
    if (n_stamps == 0) return GSB_OK;
    if (!d_leaves || !d_stamps || !d_out) return set_error(GSB_ERR_INVALID, "null argument");
    if (out_dtype != GSB_F32 && out_dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "out_dtype");
    DeviceState* st = device_state();
    if (!st->ready) return set_error(GSB_ERR_INVALID, "gsb_init has not been called");
    const cudaStream_t sm = (cudaStream_t)stream;
    // the Kolmogorov radial table for these GSParams (built once per device and GSParams)
    const double4* kolm = nullptr;
    int kolm_n = 0;
    const int rc = kolmogorov_radial(gsp, sm, &kolm, &kolm_n);
    if (rc) return rc;
    const int blocks = std::min(n_stamps, 8 * (st->sm_count > 0 ? st->sm_count : 148));
    if (out_dtype == GSB_F64)
        draw_real_kernel<double><<<blocks, 256, 0, sm>>>(n_leaves, n_stamps, *gsp, d_leaves, d_stamps, kolm, kolm_n,
                                                         static_cast<double*>(d_out), add_to_image, d_added_flux);
    else
        draw_real_kernel<float><<<blocks, 256, 0, sm>>>(n_leaves, n_stamps, *gsp, d_leaves, d_stamps, kolm, kolm_n,
                                                        static_cast<float*>(d_out), add_to_image, d_added_flux);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}
