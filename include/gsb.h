/*
 * gsb.h -- C ABI of the B200 FFT drawing path (libgsb.so).
 *
 * The reference binds its drawing path through the pybind11 module `_galsim`
 * (pysrc/module.cpp:63-111).  This library replaces the calls that
 * GSObject.drawFFT / drawKImage make through that module (galsim/gsobject.py:1927-2045,
 * 2464-2582) with batched CUDA kernels for sm_100a.  Every entry point:
 *   - is `extern "C"`, takes plain pointers and sizes, and never aborts;
 *   - returns 0 (GSB_OK) on success or a negative GSB_ERR_* code, with a message
 *     available from gsb_last_error() (reference: SBError / ImageError turned into
 *     RuntimeError by pybind11, include/galsim/SBProfile.h:49-52, include/galsim/Image.h:65-82);
 *   - takes the CUDA stream to launch on as a `void*` (a cudaStream_t, NULL = default stream);
 *   - reads and writes device memory that the caller owns, except the FT tables, which
 *     live in a gsb_tables object created and destroyed through this API.
 *
 * Units follow the reference: every profile is drawn in image coordinates (pixel = 1) after
 * the world-to-image transform, and k-space images have spacing dk = 2 pi / N.
 */
#ifndef GSB_H
#define GSB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSB_OK                0
#define GSB_ERR_INVALID      -1   /* bad argument (size, pointer, parameter range) */
#define GSB_ERR_CUDA         -2   /* a CUDA call failed */
#define GSB_ERR_UNSUPPORTED  -3   /* valid in the reference but not built here */
#define GSB_ERR_NUMERIC      -4   /* a root finder or integral did not converge */

#define GSB_MAX_OPS     32
#define GSB_MAX_LEAVES   8
#define GSB_MAX_PHASES   8
#define GSB_MAX_SCALES   8

/* Leaf profile types (reference: src/SB{Gaussian,Exponential,Sersic,Moffat,Kolmogorov,Airy,Box}.cpp). */
enum {
    GSB_GAUSSIAN    = 0,   /* p = {sigma}                                  */
    GSB_EXPONENTIAL = 1,   /* p = {r0}                                     */
    GSB_SERSIC      = 2,   /* p = {n, r0 or hlr (GSB_LEAF_SIZE_IS_HLR), trunc} */
    GSB_MOFFAT      = 3,   /* p = {beta, r0, trunc}; trunc > 0: `table` names a Moffat slot
                              built by gsb_moffat_tables_build for (beta, trunc / r0) */
    GSB_KOLMOGOROV  = 4,   /* p = {lam_over_r0}                            */
    GSB_AIRY        = 5,   /* p = {lam_over_diam, obscuration}             */
    GSB_BOX         = 6,   /* p = {width, height}                          */
    GSB_INTERPOLATED = 7   /* p = {x interpolant, k interpolant, the bits of a Lanczos k
                              interpolant's device coefficient block or 0}; `table` names an
                              image slot built by gsb_images_build (SBInterpolatedImage.cpp) */
};

/* Interpolant codes of GSB_INTERPOLATED leaves (galsim/interpolant.py, src/Interpolant.cpp). */
enum {
    GSB_INTERP_DELTA   = 0,   /* x interpolant only: uval = 1                            */
    GSB_INTERP_NEAREST = 1,
    GSB_INTERP_LINEAR  = 2,
    GSB_INTERP_CUBIC   = 3,
    GSB_INTERP_QUINTIC = 4,
    GSB_INTERP_LANCZOS = 5,   /* as x interpolant: the transform from the image's x_table
                                 (the reference's spline table of Lanczos::uCalc); as k
                                 interpolant (n <= 3): the kernel Lanczos::xCalc, with the
                                 leaf's p[2] the address of {n, conserve_dc, K_1..K_5, 0}  */
    GSB_INTERP_SINC    = 6    /* x interpolant only: uval = 1 below |u| = 1/2, 1/2 at it, 0
                                 above (SincInterpolant::uval, Interpolant.cpp:204-209)    */
};

/* Program opcodes.  A program is evaluated per k-point on a small stack of complex values:
 *   LEAF i   push leaf i's kValue at (A kx + C ky, B kx + D ky)        (SBProfile::drawK)
 *   MUL      pop b, a; push a*b                                  (Convolution._drawKImage)
 *   ADD      pop b, a; push a+b                                          (Sum._drawKImage)
 *   PHASE i  top *= fs * exp(-i (kx' cx + ky' cy)), k' from phase i's Jacobian
 *                                                   (ApplyKImagePhases, transform.py:597-599)
 *   SCALE i  top *= scale[i]                                         (transform.py:600-601) */
enum { GSB_OP_LEAF = 1, GSB_OP_MUL = 2, GSB_OP_ADD = 3, GSB_OP_PHASE = 4, GSB_OP_SCALE = 5 };

/* gsb_leaf.flags */
#define GSB_LEAF_JAC_GENERAL   1  /* Jacobian has off-diagonal terms: the reference's 2-d
                                     fillKImage rules apply (clipping differs, see
                                     SBGaussian.cpp:194-260, SBExponential.cpp:442-510) */
#define GSB_LEAF_SIZE_IS_HLR   2  /* Sersic p[1] is a half-light radius (sersic.py:224-227) */

/* gsb_phase.flags */
#define GSB_PHASE_JAC_GENERAL  1

/* Accuracy / size parameters, same meaning and order as the reference's GSParams
 * (include/galsim/GSParams.h:96-108, galsim/gsparams.py:127-135). */
typedef struct gsb_gsparams {
    int    minimum_fft_size;
    int    maximum_fft_size;
    double folding_threshold;
    double stepk_minimum_hlr;
    double maxk_threshold;
    double kvalue_accuracy;
    double xvalue_accuracy;
    double table_spacing;
    double realspace_relerr;
    double realspace_abserr;
    double integration_relerr;
    double integration_abserr;
    double shoot_accuracy;
} gsb_gsparams;

/* Topology shared by every stamp of a batch: the flattened profile tree. */
typedef struct gsb_template {
    int n_ops;
    int n_leaves;
    int n_phases;
    int n_scales;
    int op_code[GSB_MAX_OPS];
    int op_arg[GSB_MAX_OPS];
    int leaf_type[GSB_MAX_LEAVES];
} gsb_template;

/* One leaf of one stamp (device memory, stamp-major: leaves[s * n_leaves + l]). */
typedef struct gsb_leaf {
    double jac[4];     /* composed Jacobian [A, B, C, D] (row-major 2x2, transform.py:593) */
    double flux;
    double p[3];       /* profile parameters, see the type enum */
    double d[8];       /* derived values, written by gsb_prepare_leaves (GSB_INTERPOLATED and
                          truncated GSB_MOFFAT: the slot's device addresses are kept in d[6]
                          and d[7], so the leaves must be prepared again after
                          gsb_images_build / gsb_moffat_tables_build) */
    int32_t flags;     /* GSB_LEAF_* */
    int32_t table;     /* FT table slot (Sersic, truncated Moffat) or image slot (GSB_INTERPOLATED),
                          set by the caller */
} gsb_leaf;

/* One phase / flux factor of one stamp (stamp-major: phases[s * n_phases + i]). */
typedef struct gsb_phase {
    double jac[4];     /* Jacobian of the enclosing transforms (the `jac` argument of
                          Transformation._drawKImage, transform.py:592) */
    double cenx, ceny; /* shift of the Transformation */
    double flux_scaling;
    int32_t flags;     /* GSB_PHASE_* */
    int32_t pad;
} gsb_phase;

/* Geometry of one stamp (stamp-major). */
typedef struct gsb_stamp {
    int32_t N;         /* FFT size (wrap size), even; gsobject.py:1938-1955 */
    int32_t Nk;        /* k-evaluation size, even, >= N; gsobject.py:1957-1963 */
    int32_t xmin, ymin;/* stamp bounds relative to the profile centre (image view after
                          `imview._shift(-image.center)`, gsobject.py:1776) */
    int32_t nx, ny;
    int64_t out_offset;/* element offset of the stamp's (xmin, ymin) pixel in the output */
} gsb_stamp;

/* Output dtypes */
enum { GSB_F32 = 0, GSB_F64 = 1,
       /* integer image types, accepted by gsb_add_noise only */
       GSB_I16 = 2, GSB_I32 = 3, GSB_U16 = 4, GSB_U32 = 5 };

typedef struct gsb_tables gsb_tables;   /* opaque: device-resident FT tables */

/* ------------------------------------------------------------------------------------ */
const char* gsb_last_error(void);
int gsb_version(void);

/* Select the CUDA device for this thread and build the Ogata node tables on it. */
int gsb_init(int device);

/* Smallest 2^a or 3*2^a >= input (and >= 2).  Reference: goodFFTSize,
 * src/Image.cpp:1141-1153, bound at pysrc/Image.cpp:82. */
int gsb_good_fft_size(int input);

/* FT tables ---------------------------------------------------------------------------- */
int gsb_tables_create(gsb_tables** out);
int gsb_tables_destroy(gsb_tables* t);

/* Build `count` Sersic FT tables in FP64 on the device, slots 0..count-1 (replacing any
 * earlier content).  Per slot: the Hankel-transform table on a uniform ln k grid with its
 * natural-spline coefficients, the low-k quartic and high-k asymptote, maxk, stepk and the
 * half-light radius in units of r0.  Reference: SersicInfo (src/SBSersic.cpp:301-667),
 * hankel_inf (src/math/Hankel.cpp:231-249), TSpline (src/Table.cpp:553-686).
 * h_n / h_trunc_over_r0 are host arrays (h_trunc_over_r0 may be NULL: untruncated).  A slot with
 * trunc > 0 is the truncated profile's table: flux fraction, moments and the Hankel transform
 * over 0 .. trunc (math::hankel_trunc, src/math/Hankel.cpp:249-255, src/SBSersic.cpp:393-457),
 * stepk capped at trunc; its n-derivative tables (GSB_TABLES_DN) are not built. */
int gsb_sersic_tables_build(gsb_tables* t, const double* h_n, const double* h_trunc_over_r0,
                            int count, const gsb_gsparams* gsp, void* stream);

/* gsb_sersic_tables_build with options.  flags: GSB_TABLES_DN also builds, per slot, the
 * derivative of the table with respect to the Sersic index n at fixed r0 (a second Hankel
 * integrand on the same quadrature nodes, its spline, and the derivatives of the low-k and
 * high-k forms) and d ln(r_e / r0) / dn, which gsb_adjoint_images needs for Sersic leaves.
 * The tables themselves are identical with or without the flag.  No reference counterpart
 * (the reference has no derivatives). */
#define GSB_TABLES_DN 1
int gsb_sersic_tables_build_ex(gsb_tables* t, const double* h_n, const double* h_trunc_over_r0,
                               int count, const gsb_gsparams* gsp, int flags, void* stream);

/* Scale radius and flux fraction of truncated Sersic profiles (sersic.py:218-247 with
 * SersicTruncatedScale, SersicHLR and SersicIntegratedFlux, src/SBSersic.cpp:332-336, 627-775),
 * by FP64 root finding on the device.  h_in: per profile 4 doubles (n, size, trunc, flags):
 * flags bit 0 = size is a half-light radius (else the scale radius), bit 1 = flux_untruncated
 * (the half-light radius refers to the untruncated profile).  h_out: per profile (r0, flux
 * fraction inside trunc).  A half-light radius of the truncated profile needs
 * trunc > sqrt(2) hlr (GSB_ERR_INVALID otherwise, as the reference). */
int gsb_sersic_truncation(int count, const double* h_in, double* h_out, void* stream);

/* Copy slot headers back (18 doubles per slot: see gsb_tables.cu) for inspection. */
int gsb_sersic_tables_info(const gsb_tables* t, double* h_out, int count, void* stream);

/* Build `count` truncated-Moffat FT tables in FP64 on the device, Moffat slots 0..count-1
 * (replacing earlier Moffat slots; Sersic and image slots are kept).  Per slot (h_beta[i],
 * h_trunc_over_rd[i] = trunc / scale radius): the truncated Hankel transform
 *     v(k) = 2 (beta - 1) / F  int_0^t r (1 + r^2)^-beta J0(k r) dr,  F = 1 - (1 + t^2)^(1 - beta)
 * on the grid k = 0, dk, 2 dk, ... (k < 50, dk = table_spacing (kvalue_accuracy / 10)^(1/4)),
 * ended after 5 values in a row at or below kvalue_accuracy, with its natural cubic spline in
 * k^2 and maxk (in units of 1 / scale radius).  Reference: SBMoffat::setupFT
 * (src/SBMoffat.cpp:565-625), math::hankel_trunc (src/math/Hankel.cpp:249-255).  beta must be
 * > 0 and != 1 (at beta = 1 the reference's normalisation is 0 / 0); tables longer than 7264
 * nodes (kvalue_accuracy below ~2e-8 at table_spacing 1) return GSB_ERR_UNSUPPORTED. */
int gsb_moffat_tables_build(gsb_tables* t, const double* h_beta, const double* h_trunc_over_rd, int count,
                            const gsb_gsparams* gsp, void* stream);

/* Copy Moffat slot headers back, 8 doubles per slot: beta, trunc / rD, flux fraction factor F,
 * dk, nodes used, last k^2, maxk (units of 1 / rD), status. */
int gsb_moffat_tables_info(const gsb_tables* t, double* h_out, int count, void* stream);

/* Scale radius of Moffat profiles from the half-light radius (moffat.py:97-104,
 * MoffatCalculateScaleRadiusFromHLR, src/SBMoffat.cpp:103-160): h_in per profile (beta, hlr,
 * trunc), h_out the scale radius; analytic for trunc = 0, else FP64 Brent on the device.
 * trunc > 0 needs trunc > sqrt(2) hlr (GSB_ERR_INVALID); beta <= 1 has no bracket
 * (GSB_ERR_NUMERIC, as the reference's "Solve error"). */
int gsb_moffat_scale_radius(int count, const double* h_in, double* h_out, void* stream);

/* InterpolatedImage sources ------------------------------------------------------------ */
/* One image of an InterpolatedImage, placed in its zero-padded N x N frame (the reference's
 * _xim, interpolatedimage.py:590-629).  Frame coordinates X, Y run over -N/2 .. N/2-1 and the
 * frame's (0, 0) is the profile origin (the image after setCenter(0, 0)). */
typedef struct gsb_image_desc {
    int32_t N;              /* padded size, even (Image.good_fft_size of pad_factor * size) */
    int32_t nx, ny;         /* size of the nonzero region (the image, or the pad image around it) */
    int32_t x0, y0;         /* frame coordinates of the region's first pixel */
    int32_t bx0, bx1;       /* inclusive frame bounds of the image searched for the stepk   */
    int32_t by0, by1;       /*   radius (CalculateSizeContainingFlux); must contain (0, 0)  */
    int32_t x_interp;       /* GSB_INTERP_* of the x interpolant (sets the maxk scan limit)  */
    int32_t flags;          /* GSB_IMAGE_STEPK / GSB_IMAGE_MAXK: which sizes to compute     */
    int64_t pix_offset;     /* index of the region's first pixel in the packed pixel array
                               (row-major, nx pixels per row, FP64) */
    double flux;            /* flux of the nonzero region (SBInterpolatedImage::getFlux) */
    double stepk_target;    /* (1 - folding_threshold) * image flux (interpolatedimage.py:657) */
    double maxk_limit;      /* max_maxk of calculateMaxK in image units; 0 = the x
                               interpolant's 2 pi urange (SBInterpolatedImage.cpp:135-151) */
    const double* x_table;  /* GSB_INTERP_LANCZOS: device table of the x interpolant's
                               transform, 4 (n + 1) doubles: {n, mean spacing, u_0, uMax},
                               then per node {u, F(u), F''(u), 0} of a natural cubic spline
                               on equally spaced u (Lanczos::Lanczos, Interpolant.cpp:787-895);
                               NULL for the other interpolants */
} gsb_image_desc;

#define GSB_IMAGE_STEPK 1
#define GSB_IMAGE_MAXK  2
#define GSB_IMAGE_MAX_N 4096

/* Build image slots 0..count-1 of t (replacing any earlier images; Sersic slots are kept):
 * per image the half-plane DFT of its padded frame,
 *     K(p, q) = sum_XY I(X, Y) exp(-2 pi i (p X + q Y) / N),  p = 0..N/2, q = 0..N-1
 * (stored p-major),
 * in FP64 and as an FP32 copy (checkK: rfft with shift_in / shift_out, src/Image.cpp:730-812);
 * with GSB_IMAGE_STEPK the radius R = d + 1/2 of the smallest centred box holding
 * stepk_target (CalculateSizeContainingFlux, SBInterpolatedImage.cpp:1084-1110); with
 * GSB_IMAGE_MAXK maxk = (ix + 1) pi / (N / 2) for the last ring ix with |K|^2 above
 * (maxk_threshold * flux)^2 (calculateMaxK, SBInterpolatedImage.cpp:1146-1213).  Both are in
 * image units; gsb_prepare_leaves passes them on as a GSB_INTERPOLATED leaf's stepk (= R) and
 * maxk.  d_pixels is device memory; N <= GSB_IMAGE_MAX_N. */
int gsb_images_build(gsb_tables* t, int count, const gsb_image_desc* h_desc, const double* d_pixels,
                     const gsb_gsparams* gsp, void* stream);

/* Copy per image (R, maxk) back (2 doubles per image; 0 where not computed). */
int gsb_images_info(const gsb_tables* t, double* h_out, int count, void* stream);

/* Real-space drawing ----------------------------------------------------------------------- */
/* One leaf of a profile drawn in real space (drawReal: method 'no_pixel' or 'sb' on a profile
 * that is analytic in real space, gsobject.py:1810-1811, 1846-1889).  The reference walks the
 * tree with _drawReal (transform.py:571-583, sum.py:304-310), composing each Transformation's
 * Jacobian, offset and flux scaling, and draws every leaf with SBProfile::draw
 * (src/SBProfile.cpp:305-383); a gsb_xleaf holds one leaf with that composition. */
typedef struct gsb_xleaf {
    double jac[4];       /* composed Jacobian [A, B, C, D] (image = jac . profile), used when
                            flags & GSB_XLEAF_JAC */
    double xoff, yoff;   /* composed offset of the profile centre (image pixels) */
    double flux_ratio;   /* composed flux scaling |det| x flux_ratio (SBProfile::draw's flux_ratio) */
    double flux;         /* the leaf's flux */
    double p[3];         /* as gsb_leaf.p (Sersic: p[1] the scale radius; a truncated Sersic's
                            flux is that of the truncated profile); GSB_INTERPOLATED: p[0] the
                            x interpolant (GSB_INTERP_NEAREST .. GSB_INTERP_SINC) */
    int32_t type;        /* GSB_GAUSSIAN .. GSB_INTERPOLATED */
    int32_t flags;
    /* GSB_INTERPOLATED (SBInterpolatedImage::xValue, SBInterpolatedImage.cpp:167-215): the
     * nonzero region of the padded image, FP64 row-major (rnx per row) device memory, its first
     * pixel at frame position (rx0, ry0); ktab: a Lanczos interpolant's {n, conserve_dc, K_1..K_5} */
    const double* region;
    int32_t rx0, ry0, rnx, rny;
    const double* ktab;
} gsb_xleaf;

#define GSB_XLEAF_JAC 1

/* Draw n_stamps stamps of n_leaves real-space leaves each (d_leaves stamp-major): pixel (i, j)
 * of stamp s samples the sum of the leaves at image position (xmin + i, ymin + j) (the
 * stamp's bounds relative to its centre, as gsb_draw_images), each leaf's value being
 * flux_ratio x its xValue at jac^-1 ((x, y) - (xoff, yoff)) (SBGaussian.cpp:99-103,
 * SBExponential.cpp:99-103, SBSersic.cpp:92-96 and 357-361, SBMoffat.cpp:256-261,
 * SBKolmogorov.cpp:108-115 with KolmogorovInfo's radial spline, SBAiry.cpp:88-117 and
 * 410-428, SBBox.cpp:79-150), in FP64, stored as out_dtype; add_to_image adds to the output.
 * d_added_flux (optional) receives per stamp the FP64 sum of the drawn (rounded) values. */
int gsb_draw_real(int n_leaves, int n_stamps, const gsb_gsparams* gsp, const gsb_xleaf* d_leaves,
                  const gsb_stamp* d_stamps, void* d_out, int out_dtype, int add_to_image,
                  double* d_added_flux, void* stream);

/* Chromatic drawing ---------------------------------------------------------------------- */
/* The wavelength integral of chromatic drawing (the integrators' IntegrationRule.__call__,
 * galsim/integ.py:134-146): out[p] = sum_s w[s] * stamp_s[p] over n_stamps stamps of npix
 * pixels each, stamp s starting at element d_offsets[s] of d_flat (the monochromatic images
 * drawn at the integration wavelengths, e.g. one gsb_draw_images batch); FP64 accumulation,
 * in / out dtypes GSB_F32 or GSB_F64.  All pointers are device memory. */
int gsb_weighted_stamp_sum(const void* d_flat, int in_dtype, const int64_t* d_offsets,
                           const double* d_weights, int n_stamps, int64_t npix, void* d_out,
                           int out_dtype, void* stream);

/* Noise ---------------------------------------------------------------------------------- */
/* GaussianNoise, PoissonNoise and CCDNoise applied to stamps in device memory with the
 * reference's random streams (galsim/noise.py:259-263, 331-356, 463-486; src/Random.cpp).  Each
 * stamp has its own BaseDeviate(seed) (Random.cpp:156-191: the seed passes through an mt11213b
 * whose third draw seeds the mt19937), positioned `skip` raw 32-bit draws into its stream
 * (0 for a fresh BaseDeviate); the deviates follow Boost.Random 1.48 as the reference vendors it
 * (uniform_01, Box-Muller normal pairs, inversion / PTRD Poisson). */
enum { GSB_NOISE_GAUSSIAN = 0, GSB_NOISE_POISSON = 1, GSB_NOISE_CCD = 2, GSB_NOISE_VARIABLE_GAUSSIAN = 3,
       GSB_NOISE_UNIFORM = 4 };

typedef struct gsb_noise_stamp {
    int64_t offset;    /* first pixel of the stamp in the image buffer (elements) */
    int32_t npix;      /* pixels, row-major and contiguous */
    int32_t pad;
    int64_t seed;      /* the BaseDeviate seed (nonzero) */
    int64_t skip;      /* raw draws of that stream already consumed */
} gsb_noise_stamp;

typedef struct gsb_noise_params {
    double sigma;          /* GaussianNoise sigma */
    double sky_level;      /* Poisson / CCD: sky added before the draw */
    double gain;           /* CCD gain (e- / ADU); ignored for Poisson */
    double read_noise;     /* CCD read noise (e-) */
    double frac_sky;       /* subtracted in FP64 before the cast to the image type */
    double int_sky;        /* subtracted after the cast (the reference's numpy scalar rules
                              decide the split; for float images frac_sky is 0) */
    int32_t int_sky_same_dtype;   /* int_sky has the image's type: subtract in that type */
    int32_t pad;
} gsb_noise_params;

/* Add noise of `kind` to n_stamps stamps of d_image (GSB_F32, GSB_F64, or an integer type:
 * GSB_I16 / I32 / U16 / U32, cast as numpy's unsafe cast does on the reference's host --
 * truncation toward zero, wrapping to the type's width); max_npix bounds the
 * stamps' pixel counts.  Poisson and CCD noise need d_scratch (one double per pixel, addressed
 * like d_image) and d_used.  GSB_NOISE_VARIABLE_GAUSSIAN (VariableGaussianNoise, noise.py:590-636,
 * Random.cpp:402-450) reads each pixel's variance from d_scratch (FP64, addressed like d_image,
 * left unchanged) and adds unit deviates times its square root; p->sigma is ignored.
 * GSB_NOISE_UNIFORM adds uniform deviates in [0, 1), one 32-bit word each (UniformDeviate,
 * boost uniform_01: word / 2^32), the deviates of the product's UniformDeviate and DeviateNoise.  d_used (may be NULL for Gaussian noise) receives, per stamp, the raw
 * draws consumed since seeding (skip + this call's draws), so a caller can continue the stream.
 * Gaussian: one warp per stamp.  Poisson / CCD: the expectations in parallel, then one warp per
 * stamp walks its sequential stream (speculative draws of 32 pixels at once, committed up to the
 * first whose count of draws was mispredicted), then the read noise and the cast one warp per
 * stamp.  No allocation. */
int gsb_add_noise(int kind, const gsb_noise_params* p, const gsb_noise_stamp* d_stamps, int n_stamps,
                  int max_npix, void* d_image, int dtype, double* d_scratch, long long* d_used,
                  void* stream);

/* FITS file images ---------------------------------------------------------------------- */
/* One HDU of a FITS file assembled on the device (the layout galsim/fits.py writes through
 * astropy: FITS Standard 4.0 header blocks and big-endian data padded to 2880 bytes). */
typedef struct gsb_fits_hdu {
    int64_t header_src;   /* byte offset of the HDU's header in d_headers (multiple of 16) */
    int64_t header_len;   /* header bytes: formatted cards padded to a multiple of 2880 */
    int64_t data_src;     /* element offset of the HDU's first pixel in d_src */
    int64_t n_elem;       /* pixels, in the order they are stored (row-major, stamps in turn) */
    int64_t dst;          /* byte offset of the HDU in d_out (multiple of 2880, ascending) */
} gsb_fits_hdu;

/* Write the file image of n_hdus HDUs (host records h_hdus, checked against the buffer sizes)
 * into d_out: each header copied, the pixels of d_src (GSB_F32 / GSB_F64) byte-swapped to
 * big-endian after it, and the data zero-padded to a 2880-byte block.  d_headers and d_out are
 * 16-byte aligned.  Replaces astropy's HDUList.writeto as called by fits.py:378-701 for the
 * pixels; the file itself is written by the caller from the copied-back buffer. */
int gsb_fits_pack(const gsb_fits_hdu* h_hdus, int n_hdus, const void* d_headers, long long header_bytes,
                  const void* d_src, long long src_elems, int dtype, void* d_out, long long out_bytes,
                  void* stream);

/* Leaves -------------------------------------------------------------------------------- */
/* Fill the derived values of every leaf and write its stepk and maxk (d_info[2*(s*L+l)]).
 * Reference: the leaf constructors and stepK()/maxK() (SBGaussian.cpp:55-89,
 * SBExponential.cpp:65-92 and 513-554, SBSersic.cpp:71-90 and 301-324,
 * SBMoffat.cpp:163-244 and 481-549, SBKolmogorov.cpp:84-100 and 338-420,
 * SBAiry.cpp:66-81 and 332-445, SBBox.cpp:40-60) and the Python overrides
 * (gaussian.py:148-155, exponential.py:131-132, kolmogorov.py:281-284, airy.py:217-219,
 * box.py:100-106).  Sersic leaves must already name a built table slot. */
int gsb_prepare_leaves(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                       gsb_leaf* d_leaves, const gsb_tables* t, double* d_info, void* stream);

/* Drawing -------------------------------------------------------------------------------- */
/* Scratch bytes gsb_draw_images needs for a bucket of stamps that all have FFT size N. */
size_t gsb_draw_workspace_size(int N, int n_stamps, int precision);

/* drawImage(method='fft') for a bucket of stamps that share one FFT size N:
 * k-space evaluation of the program at the Nk x Nk grid points, Hermitian wrap onto N,
 * c2r inverse FFT, crop into the stamp, cast, optional add, and the stamp's flux sum.
 * Reference: drawFFT_makeKImage / _drawKImage / drawFFT_finish (gsobject.py:1927-2045)
 * with wrapImage (src/Image.cpp:578-727) and irfft (src/Image.cpp:815-912).
 * precision: GSB_F32 or GSB_F64 arithmetic.  d_added_flux (may be NULL): per stamp,
 * the compensated sum of the drawn pixels (gsobject.py:2011). */
int gsb_draw_images(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                    const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                    const gsb_stamp* d_stamps, const gsb_tables* t,
                    void* d_out, int out_dtype, int add_to_image, double* d_added_flux,
                    int precision, void* d_workspace, size_t workspace_bytes, void* stream);

/* gsb_draw_images for a bucket whose FFT size N the caller passes (every stamp's N must equal
 * it): no host synchronisation, so buckets can run concurrently on several streams and the
 * call can be captured in a CUDA graph (after a first call with the same N and precision,
 * which may set up device state).  Same contract as gsb_draw_images otherwise. */
int gsb_draw_bucket(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                    const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                    const gsb_stamp* d_stamps, const gsb_tables* t, int N,
                    void* d_out, int out_dtype, int add_to_image, double* d_added_flux,
                    int precision, void* d_workspace, size_t workspace_bytes, void* stream);

/* Reorders device records between the caller's stamp order and the FFT-size bucket order that
 * gsb_draw_bucket draws (stamps sorted by N, each bucket contiguous), replacing the per-object
 * order of drawFFT calls (gsobject.py:2014-2045) with one launch: scatter = 0 gathers
 * dst[i] = src[perm[i]] (leaf, phase and scale records into bucket order); scatter = 1 scatters
 * dst[perm[i]] = src[i] (per-stamp results such as the added flux back to the caller's order).
 * count records of record_bytes (a multiple of 8) each; d_dst, d_src and d_perm 8-byte aligned,
 * d_dst not aliasing d_src.  Entries of d_perm outside [0, count) are skipped.  Asynchronous on
 * `stream`; no allocation, graph-capturable. */
int gsb_permute_records(void* d_dst, const void* d_src, const int64_t* d_perm, int64_t count,
                        int64_t record_bytes, int scatter, void* stream);

/* Kernel variant for buckets of FFT size N <= 1024: 0 = automatic (default), 1 = always the
 * fused one-CTA-per-stamp kernel, 2 = the split column/row kernels where N >= 192.  In automatic
 * mode the first draw of each (device, precision, N, floor(log2 stamps)) class with fewer than
 * 2 stamps per SM times both on its inputs (when it overwrites its output and the stream is
 * not being captured) and keeps the faster; the choice then holds for the process.  Results of
 * the two variants agree to floating-point rounding.  No reference counterpart. */
int gsb_draw_set_variant(int variant);

/* The FP64 exponential that the Hankel quadratures of the table stage use (table-driven,
 * after P. T. P. Tang, ACM TOMS 15 (1989) 144-157), applied to n device values; exposed so that
 * its accuracy can be checked against the CUDA math library.  No reference counterpart. */
int gsb_exp_fp64(const double* d_x, double* d_y, int n, void* stream);

/* The same with the table size chosen: 32 (gsb_exp_fp64) or 256, the variant with a degree-4
 * polynomial that the Sersic quadrature kernel uses. */
int gsb_exp_fp64_ex(const double* d_x, double* d_y, int n, int table_size, void* stream);

/* Text report of the tuned classes, one line each; returns its length (writes at most len-1
 * characters and a terminating zero to buf when buf is not NULL). */
int gsb_draw_tune_report(char* buf, size_t len);

/* drawKImage: evaluate the program on an (nkx x nky) grid of k points
 * kx = (kxmin + i) dk, ky = (kymin + j) dk, into complex output (interleaved re, im) with
 * row stride nkx.  One grid per stamp, stamp s at d_out + s * nkx * nky complex elements.
 * Reference: GSObject.drawKImage / _drawKImage (gsobject.py:2464-2582). */
int gsb_draw_kimages(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                     const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                     const gsb_tables* t, double dk, int kxmin, int kymin, int nkx, int nky,
                     void* d_out, int out_dtype, void* stream);

/* The reference's compiled hot-path steps one by one --------------------------------------
 * For callers that keep the reference's Python orchestration (GSObject.drawFFT,
 * galsim/gsobject.py:2014-2045, and the _drawKImage tree walk) and replace only what it calls
 * in _galsim.  Each acts on one image in device memory; gsb_draw_images fuses all four. */

/* SBProfile.drawK (pysrc/SBProfile.cpp:35-40, src/SBProfile.cpp:383-425): the profile's
 * k-values on the grid kx = i dk, ky = j dk for the image bounds i = xmin .. xmin+nx-1,
 * j = ymin .. ymin+ny-1, written as complex (re, im) rows of nx values, FP32 or FP64 per
 * out_dtype; n_stamps images one after the other.  jac (a host array of 4 doubles, row-major
 * [A, B, C, D], or NULL) is the drawK Jacobian: as in Transformation._drawKImage
 * (transform.py:592) it multiplies every leaf's and phase's composed Jacobian from the left,
 * and the 1-d / 2-d fill rules follow the product.  The records are the batch records of
 * gsb_draw_kimages (prepared by gsb_prepare_leaves). */
int gsb_draw_k(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp, const gsb_leaf* d_leaves,
               const gsb_phase* d_phases, const double* d_scales, const gsb_tables* t, double dk,
               const double* jac, int xmin, int ymin, int nx, int ny, void* d_out, int out_dtype,
               void* stream);

/* ApplyKImagePhases (pysrc/SBTransform.cpp:27-40, src/SBTransform.cpp:740-883): multiply the
 * complex k-image (bounds xmin.., ymin.., nx x ny, row stride `stride` complex elements,
 * complex64 for GSB_F32 or complex128 for GSB_F64) in place by
 * flux_scaling * exp(-i (kx' cenx + ky' ceny)), kx = i dk, ky = j dk, (kx', ky') =
 * (A kx + C ky, B kx + D ky) from jac (host, 4 doubles, or NULL for the identity).  The phase
 * is formed in FP64 turns. */
int gsb_apply_kimage_phases(void* d_image, int dtype, int xmin, int ymin, int nx, int ny, long long stride,
                            double dk, const double* jac, double cenx, double ceny, double flux_scaling,
                            void* stream);

/* wrapImage (pysrc/Image.cpp:60-61, src/Image.cpp:578-727, Image.wrap in image.py:711-796):
 * fold the image with bounds (xmin..xmax, ymin..ymax) (row stride in_stride elements) onto
 * the bounds b = (bxmin..bxmax, bymin..bymax): every cell of b receives the sum of its aliases
 * (periods of b's widths).  hermx: the image holds x >= 0 only and is Hermitian
 * (X(-x, -y) = conj X(x, y)); the x period is 2 bxmax; the reference's conditions apply
 * (xmin = bxmin = 0, symmetric y bounds, b missing its most negative row).  Real (is_complex
 * = 0) or complex images, FP32 or FP64 per dtype.  Unlike the reference, which wraps in place
 * and returns the subimage, the result is written to d_out (b's cells, row stride
 * out_stride), which must not overlap d_in.  hermy returns GSB_ERR_UNSUPPORTED. */
int gsb_wrap_image(const void* d_in, int dtype, int is_complex, int xmin, int xmax, int ymin, int ymax,
                   long long in_stride, int bxmin, int bxmax, int bymin, int bymax, int hermx, int hermy,
                   void* d_out, long long out_stride, void* stream);

/* irfft (pysrc/Image.cpp:53-57, src/Image.cpp:815-912): inverse real FFT of the Hermitian
 * half plane with bounds (0..Nx/2, -Ny/2..Ny/2-1) (complex64 or complex128 per in_dtype, row
 * stride in_stride complex elements) into FP64 rows of the output bounds
 * (-Nx/2..Nx/2+1, -Ny/2..Ny/2-1), row stride out_stride >= Nx + 2 doubles (the last two columns
 * of each row are not written).  Scaled by 1/(Nx Ny); shift_in swaps the ky halves into FFT
 * order, shift_out multiplies by (-1)^(i+j) so that x = y = 0 lands at the centre, as the
 * reference's flags do.  As in a c2r transform, the imaginary parts left in the kx = 0 and
 * kx = Nx/2 columns after the y transform are ignored.  Nx, Ny: 2^a or 3*2^a up to 12288
 * (others return GSB_ERR_UNSUPPORTED).  d_work: gsb_irfft_workspace_size(Nx, Ny) bytes of
 * device scratch. */
int gsb_irfft(const void* d_in, int in_dtype, int Nx, int Ny, long long in_stride, double* d_out,
              long long out_stride, int shift_in, int shift_out, void* d_work, size_t work_bytes,
              void* stream);
size_t gsb_irfft_workspace_size(int Nx, int Ny);

/* gsb_draw_images without any device allocation.  This entry point has no counterpart in
 * the reference; it exists for callers that cannot allocate device memory while they draw
 * (an application that owns a fixed GPU memory budget, or a plugin inside another program's
 * memory pool).  Same inputs and outputs as gsb_draw_images for one FFT-size bucket
 * (InterpolatedImage leaves included), with the bucket's FFT size N passed explicitly
 * (32 <= N <= 1024, 2^a or 3*2^a; larger N returns GSB_ERR_UNSUPPORTED).  Every stamp's N
 * must equal N: a check on the device compares them before the draw and a mismatch returns
 * GSB_ERR_INVALID (the call reads that check back, so it returns once the stream has reached
 * it).  The scratch that gsb_draw_images takes from the caller comes instead from a 32 MiB
 * array compiled into the library (held by every GPU that loads it until exit).  The first
 * call on a device looks up that array's address and should come before any stream capture;
 * the address is kept, so do not use the library on a device after cudaDeviceReset.  All
 * calls share the array: calls that overlap on the GPU race, so serialise them on one
 * stream. */
int gsb_draw_images_noalloc(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                            const gsb_leaf* d_leaves, const gsb_phase* d_phases,
                            const double* d_scales, const gsb_stamp* d_stamps,
                            const gsb_tables* t, int N, void* d_out, int out_dtype,
                            int add_to_image, double* d_added_flux, int precision, void* stream);

/* Adjoint ------------------------------------------------------------------------------ */
/* Gradient entries per stamp for this template, in this order:
 *   per leaf l   (6): d/dflux, d/djac[0..3], d/dp[0] (Sersic n, else 0)
 *   per phase i  (7): d/dcenx, d/dceny, d/dflux_scaling, d/djac[0..3]
 *   per scale i  (1): d/dscale
 * Returns the count (>= 6) or a negative GSB_ERR_* code.  Size parameters have no entry of
 * their own: each leaf depends on its size s and Jacobian J only through s J, so
 * d/d(ln s) = sum_ij J_ij d/dJ_ij (Box: width with J[0], J[2]; height with J[1], J[3]).
 * For a Sersic leaf with GSB_LEAF_SIZE_IS_HLR the n entry is at fixed half-light radius. */
int gsb_adjoint_grad_count(const gsb_template* tpl);

/* Scratch bytes gsb_adjoint_images needs for a bucket of stamps of FFT size N. */
size_t gsb_adjoint_workspace_size(int N, int n_stamps, int precision);

/* Reverse mode of gsb_draw_images for one FFT-size bucket (N in 32..16384; above 1024 the split
 * row / column kernels of the large draw path in reverse, with per-stamp slabs in the
 * workspace): given
 * d_cotangent = dL/d(image), laid out exactly as the images gsb_draw_images writes for the same
 * stamps (out_offset, nx, ny; dtype cot_dtype), write d_grad[s * count + e] = dL/d(entry e of
 * stamp s) (FP64, count from gsb_adjoint_grad_count).  The derivatives are analytic (each
 * profile's dkValue/dparameter, the phase and the products of the program) and are taken on
 * the stamp's fixed grid (N, Nk); clipped k-points contribute zero.  Sersic leaves need tables
 * built with GSB_TABLES_DN.  No reference counterpart (the reference has no derivatives); it
 * is the adjoint of gsobject.py:1927-2045 + src/Image.cpp:578-912 for fixed sizes.
 * want_mask names the records to differentiate (leaf l: bit l, phase p: bit 8 + p, scale q:
 * bit 16 + q; GSB_WANT_ALL for every record); the entries of the others are written as 0 and
 * their factors are folded into per-stamp 1-d tables, which makes the pass cheaper. */
#define GSB_WANT_ALL 0xffffffffu
int gsb_adjoint_images(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                       const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                       const gsb_stamp* d_stamps, const gsb_tables* t, int N,
                       const void* d_cotangent, int cot_dtype, double* d_grad, unsigned int want_mask,
                       int precision, void* d_workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GSB_H */
