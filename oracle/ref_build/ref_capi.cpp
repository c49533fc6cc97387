// ORACLE-ONLY: a plain C ABI over the reference's own C++ objects (compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libgsref.so).  It exposes exactly
// the reference calls that GSObject.drawFFT makes (galsim/gsobject.py:1927-2045):
//   SBProfile::drawK          (pysrc/SBProfile.cpp:35-40, src/SBProfile.cpp:383-425)
//   ApplyKImagePhases         (pysrc/SBTransform.cpp:27-40, src/SBTransform.cpp:843-883)
//   wrapImage                 (pysrc/Image.cpp:60-61, src/Image.cpp:578-727)
//   irfft                     (pysrc/Image.cpp:53-57, src/Image.cpp:815-912)
//   goodFFTSize               (pysrc/Image.cpp:82, src/Image.cpp:1141-1153)
//   stepK / maxK of the leaf profiles and SersicHLR
// so that the drawFFT orchestration, restated in oracle/ref_draw.py, runs on the
// reference's own arithmetic without the reference Python package.  Used only by tests
// and by the CPU baseline arm of bench.py.
#include <complex>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "GSParams.h"
#include "Image.h"
#include "SBAiry.h"
#include "SBBox.h"
#include "SBExponential.h"
#include "SBGaussian.h"
#include "SBInterpolatedImage.h"
#include "Interpolant.h"
#include "Random.h"
#include "SBKolmogorov.h"
#include "SBMoffat.h"
#include "SBSersic.h"
#include "SBTransform.h"

using namespace galsim;

namespace {

thread_local std::string g_err;

GSParams make_gsp(const double* g)
{
    return GSParams(int(g[0]), int(g[1]), g[2], g[3], g[4], g[5], g[6], g[7], g[8], g[9],
                    g[10], g[11], g[12]);
}

// Profile type codes shared with oracle/ref_draw.py.
enum { GAUSS = 0, EXPO = 1, SERSIC = 2, MOFFAT = 3, KOLMO = 4, AIRY = 5, BOX = 6 };

std::unique_ptr<SBProfile> make_profile(int type, const double* p, double flux, const GSParams& gsp)
{
    switch (type) {
      case GAUSS: return std::unique_ptr<SBProfile>(new SBGaussian(p[0], flux, gsp));
      case EXPO: return std::unique_ptr<SBProfile>(new SBExponential(p[0], flux, gsp));
      case SERSIC: return std::unique_ptr<SBProfile>(new SBSersic(p[0], p[1], flux, p[2], gsp));
      case MOFFAT: return std::unique_ptr<SBProfile>(new SBMoffat(p[0], p[1], p[2], flux, gsp));
      case KOLMO: return std::unique_ptr<SBProfile>(new SBKolmogorov(p[0], flux, gsp));
      case AIRY: return std::unique_ptr<SBProfile>(new SBAiry(p[0], p[1], flux, gsp));
      case BOX: return std::unique_ptr<SBProfile>(new SBBox(p[0], p[1], flux, gsp));
    }
    throw std::runtime_error("unknown profile type");
}

template <typename T>
ImageView<T> view(T* data, int xmin, int xmax, int ymin, int ymax)
{
    ptrdiff_t ncol = xmax - xmin + 1, nrow = ymax - ymin + 1;
    shared_ptr<T> owner;
    return ImageView<T>(data, data + ncol * nrow, ncol * nrow, owner, 1, int(ncol),
                        Bounds<int>(xmin, xmax, ymin, ymax));
}

std::unique_ptr<Interpolant> make_interp(int code, const GSParams& gsp)
{
    switch (code) {
      case 0: return std::unique_ptr<Interpolant>(new Delta(gsp));
      case 1: return std::unique_ptr<Interpolant>(new Nearest(gsp));
      case 2: return std::unique_ptr<Interpolant>(new Linear(gsp));
      case 3: return std::unique_ptr<Interpolant>(new Cubic(gsp));
      case 4: return std::unique_ptr<Interpolant>(new Quintic(gsp));
    }
    throw std::runtime_error("unknown interpolant");
}

// An SBInterpolatedImage with the buffers it views (InterpolatedImage._sbp,
// galsim/interpolatedimage.py:481-500).
struct IIHandle {
    GSParams gsp;
    std::vector<double> data;
    std::unique_ptr<Interpolant> xi, ki;
    std::unique_ptr<SBInterpolatedImage> sb;
    explicit IIHandle(const GSParams& g) : gsp(g) {}
};

}  // namespace

extern "C" {

// SBInterpolatedImage over an N x N padded image (bounds -N/2..N/2-1 both ways), with the
// image and nonzero bounds as (xmin, xmax, ymin, ymax); stepk / maxk <= 0 are computed.
void* gsref_ii_create(const double* xim, int N, const int* ib, const int* nb, int xcode, int kcode,
                      double stepk, double maxk, const double* gsp)
{
    try {
        std::unique_ptr<IIHandle> h(new IIHandle(make_gsp(gsp)));
        h->data.assign(xim, xim + size_t(N) * N);
        h->xi = make_interp(xcode, h->gsp);
        h->ki = make_interp(kcode, h->gsp);
        ImageView<double> im = view(h->data.data(), -N / 2, N / 2 - 1, -N / 2, N / 2 - 1);
        h->sb.reset(new SBInterpolatedImage(im, Bounds<int>(ib[0], ib[1], ib[2], ib[3]),
                                            Bounds<int>(nb[0], nb[1], nb[2], nb[3]), *h->xi, *h->ki,
                                            stepk, maxk, h->gsp));
        return h.release();
    } catch (std::exception& e) { g_err = e.what(); return nullptr; }
}

void gsref_ii_destroy(void* h) { delete static_cast<IIHandle*>(h); }

// calculateMaxK(max_maxk) then maxK() (image units).
int gsref_ii_maxk(void* h, double max_maxk, double* out)
{
    try {
        IIHandle* ii = static_cast<IIHandle*>(h);
        ii->sb->calculateMaxK(max_maxk);
        *out = ii->sb->maxK();
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

int gsref_ii_draw_k(void* h, double* kimage, int xmin, int xmax, int ymin, int ymax, double dk,
                    const double* jac)
{
    try {
        IIHandle* ii = static_cast<IIHandle*>(h);
        double j[4];
        if (jac) std::memcpy(j, jac, sizeof(j));
        ii->sb->drawK(view(reinterpret_cast<std::complex<double>*>(kimage), xmin, xmax, ymin, ymax),
                      dk, jac ? j : nullptr);
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

// CCDNoise._applyTo (galsim/noise.py:463-486) on a float64 image with the reference's
// deviates: Poisson in electrons from a fresh BaseDeviate(seed), then the Gaussian read noise
// from the same stream (for the CPU baseline of the noise stage).
int gsref_ccd_noise(double* img, long long n, long seed, double sky, double gain, double read_noise)
{
    try {
        BaseDeviate rng(seed);
        PoissonDeviate pd(rng, 1.);
        for (long long i = 0; i < n; ++i) {
            double v = img[i] + sky;
            v *= gain;
            img[i] = v < 0. ? 0. : v;
        }
        pd.generateFromExpectation(n, img);
        for (long long i = 0; i < n; ++i) img[i] /= gain;
        if (read_noise > 0.) {
            GaussianDeviate gd(rng, 0., read_noise / gain);
            gd.clearCache();
            gd.addGenerate(n, img);
        }
        for (long long i = 0; i < n; ++i) img[i] -= sky;
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

// CalculateSizeContainingFlux on an image with bounds (xmin, xmax, ymin, ymax).
int gsref_size_containing_flux(double* im, int xmin, int xmax, int ymin, int ymax, double target,
                               double* out)
{
    try {
        *out = CalculateSizeContainingFlux(view(im, xmin, xmax, ymin, ymax), target);
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

const char* gsref_last_error() { return g_err.c_str(); }

int gsref_good_fft_size(int n) { return goodFFTSize(n); }

// out[0] = stepK, out[1] = maxK of one leaf profile.
int gsref_profile_info(int type, const double* p, double flux, const double* gsp, double* out)
{
    try {
        auto prof = make_profile(type, p, flux, make_gsp(gsp));
        out[0] = prof->stepK();
        out[1] = prof->maxK();
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

// SBProfile::drawK into a complex128 image with the given bounds; jac may be NULL.
int gsref_draw_k(int type, const double* p, double flux, const double* gsp, double* kimage,
                 int xmin, int xmax, int ymin, int ymax, double dk, const double* jac)
{
    try {
        auto prof = make_profile(type, p, flux, make_gsp(gsp));
        double j[4];
        if (jac) std::memcpy(j, jac, sizeof(j));
        prof->drawK(view(reinterpret_cast<std::complex<double>*>(kimage), xmin, xmax, ymin, ymax),
                    dk, jac ? j : nullptr);
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

int gsref_apply_phases(double* kimage, int xmin, int xmax, int ymin, int ymax, double dk,
                       const double* jac, double cenx, double ceny, double flux_scaling)
{
    try {
        ApplyKImagePhases(view(reinterpret_cast<std::complex<double>*>(kimage), xmin, xmax, ymin, ymax),
                          dk, jac, cenx, ceny, flux_scaling);
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

int gsref_wrap(double* kimage, int xmin, int xmax, int ymin, int ymax,
               int bxmin, int bxmax, int bymin, int bymax, int hermx, int hermy)
{
    try {
        wrapImage(view(reinterpret_cast<std::complex<double>*>(kimage), xmin, xmax, ymin, ymax),
                  Bounds<int>(bxmin, bxmax, bymin, bymax), hermx != 0, hermy != 0);
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

// kimage: the wrapped sub-image (bounds 0..N/2, -N/2..N/2-1) given by its base pointer and
// the full row stride (in complex elements) of the array it lives in.
int gsref_irfft(const double* kimage, int kstride, int N, double* out)
{
    try {
        shared_ptr<std::complex<double> > kowner;
        const std::complex<double>* k = reinterpret_cast<const std::complex<double>*>(kimage);
        ptrdiff_t n = ptrdiff_t(kstride) * N;
        ConstImageView<std::complex<double> > in(
            const_cast<std::complex<double>*>(k), k + n, n, kowner, 1, kstride,
            Bounds<int>(0, N / 2, -N / 2, N / 2 - 1));
        irfft(in, view(out, -N / 2, N / 2 + 1, -N / 2, N / 2 - 1), true, true);
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return -1; }
}

double gsref_sersic_hlr(double n, double flux_fraction) { return SersicHLR(n, flux_fraction); }

}  // extern "C"
