// Internal definitions shared by the libgsb translation units.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string>

#include "gsb.h"
#include "gsb_math.cuh"

namespace gsb {

// Records the message for gsb_last_error() and returns the code.
int set_error(int code, const std::string& msg);

// Host-side checks shared by the entry points: a template's sizes, program (stack discipline,
// indices) and leaf types; an FFT size of the form 2^a or 3 * 2^a.
int validate_template(const gsb_template* tpl);
bool good_fft_size_ok(int n);

#define GSB_CUDA_CHECK(expr)                                                              \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            (void)cudaGetLastError(); /* clear a non-sticky error for the next call */    \
            return ::gsb::set_error(GSB_ERR_CUDA, std::string(#expr) + ": " +            \
                                    cudaGetErrorString(e_));                              \
        }                                                                                 \
    } while (0)

// One leaf as used inside kernels (gsb_leaf plus its type).
struct LeafParams {
    double jac[4];
    double flux;
    double d[8];
    int flags;
    int table;
    int type;
};

// Sersic FT table slot: header plus nodes (arg - front, value, y2, 0).
// Header layout (doubles): see kSersicHeader* below.
struct SersicTableView {
    int n;              // number of nodes in the spline
    double front, da;   // first arg, equal-spacing step for the index lookup
    double ksq_min, ksq_max, kderiv2, kderiv4, highk_a, highk_b;
    const double4* node;
};

enum {
    kSH_N = 0, kSH_NUSED, kSH_FRONT, kSH_DA, kSH_KSQMIN, kSH_KSQMAX, kSH_KD2, kSH_KD4,
    kSH_HIGHA, kSH_HIGHB, kSH_MAXK, kSH_STEPK, kSH_RE, kSH_DLOGK, kSH_NCAND, kSH_STATUS,
    kSH_TRUNC, kSH_FLUXFRAC,    // truncation radius / r0 (0: untruncated) and the flux fraction within it
    kSersicHeader = 18
};

// Truncated Moffat FT table slot (SBMoffat::setupFT, src/SBMoffat.cpp:565-625): header plus
// nodes (k^2, value, y2, 0) of a natural cubic spline in k^2 on the grid k = 0, dk, 2 dk, ...
// (k in units of 1 / rD; the grid is the reference's running sum k += dk).
enum {
    kMH_BETA = 0, kMH_TRUNC, kMH_FLUXFACTOR, kMH_DK, kMH_NUSED, kMH_KSQMAX, kMH_MAXK, kMH_STATUS,
    kMoffatHeader = 8
};

// Per-slot derivative header (doubles) of tables built with n-derivatives: d/dn (at fixed
// r0) of the low-k coefficients and of the high-k fit, and d ln(r_e / r0) / dn.
// The table's grid starts at front = ln k_min(n) - 0.001, so its nodes k_i move with n:
// node derivatives are total derivatives along k_i(n), and dfront/dn is kept to shift the
// spline argument.
enum {
    kSD_DKD2 = 0, kSD_DKD4, kSD_DHIGHA, kSD_DHIGHB, kSD_DLNRE, kSD_DFRONT,
    kSersicDHeader = 8
};

// d/dn of a Sersic table: spline nodes (x, dy/dn, d2y/dn, 0) on the table's own x grid.
struct SersicDnView {
    double dkd2, dkd4, dhigha, dhighb, dlnre, dfront;
    const double4* node;
};

// The reference k-image grid a point belongs to (for clip rules that depend on the grid).
struct GridRef {
    double dk;
    int x0, y0;   // integer k index of column 0 / row 0
    int m, n;     // columns, rows
};

// Airy annulus autocorrelation (SBAiry.cpp:259-329 obscured, :395-408 unobscured);
// t = k^2 / (pi D)^2.
template <typename T>
__device__ inline T airy_chord(T r, T h, T rsq, T hsq)
{
    if (r == T(0)) return T(0);
    // Clamps keep rounding at the overlap boundaries inside the domains of asin / sqrt.
    return rsq * asin(fmin(h / r, T(1))) - h * sqrt(fmax(rsq - hsq, T(0)));
}

template <typename T>
__device__ inline T airy_circle_same(T r, T rsq, T tsq)
{
    if (tsq >= T(4) * rsq) return T(0);
    if (tsq == T(0)) return T(kPi) * rsq;
    const T hsq = fmax(rsq - tsq / T(4), T(0));
    const T h = sqrt(hsq);
    return T(2) * airy_chord<T>(r, h, rsq, hsq);
}

template <typename T>
__device__ inline T airy_circle_two(T r, T s, T rsq, T ssq, T tsq)
{
    const T rps_sq = (r + s) * (r + s);
    if (tsq >= rps_sq) return T(0);
    const T rms_sq = (r - s) * (r - s);
    if (tsq <= rms_sq) return T(kPi) * ssq;
    const T hsq = fmax(T(0.5) * (rsq + ssq) - (tsq * tsq + rps_sq * rms_sq) / (T(4) * tsq), T(0));
    const T h = sqrt(hsq);
    if (tsq < rsq - ssq)
        return T(kPi) * ssq - airy_chord<T>(s, h, ssq, hsq) + airy_chord<T>(r, h, rsq, hsq);
    return airy_chord<T>(s, h, ssq, hsq) + airy_chord<T>(r, h, rsq, hsq);
}

// FP32 lens areas in a form without the reference's asin(h / r) near h = r.  For two discs
// (radii r, s) with centres d apart, the common chord lies a_r = (d^2 + r^2 - s^2) / (2d)
// from the r-centre and a_s = d - a_r from the s-centre, with half length h, and
//     A = r^2 atan2(h, a_r) + s^2 atan2(h, a_s) - d h,
// which covers the minor and the major segment (a < 0) alike and is stationary in h and
// a_r, so their rounding does not reach A to first order.  The reference's form takes
// asin of h / r -> 1 at small d, where an FP32 h = sqrt(1 - d^2/4) rounds to 1 and drops
// the -2 d r term of A: a relative error up to ~2 d / pi on the innermost k rings, which on
// grids with dk ~ 5e-4 (N >= 6144) biased the drawn flux by 1e-5 .. 1e-4.  FP64 keeps the
// reference's form (its rounding there is ~1e-13 of the value).
template <typename T>
__device__ inline T airy_lens_same_f32(T rsq, T tsq)
{
    if (tsq >= T(4) * rsq) return T(0);
    if (tsq == T(0)) return T(kPi) * rsq;
    const T d = sqrt(tsq);
    const T h = sqrt(fmax(rsq - tsq / T(4), T(0)));
    return T(2) * rsq * atan2(h, T(0.5) * d) - d * h;
}

template <typename T>
__device__ inline T airy_lens_two_f32(T r, T s, T rsq, T ssq, T tsq)
{
    const T rps_sq = (r + s) * (r + s);
    if (tsq >= rps_sq) return T(0);
    const T rms_sq = (r - s) * (r - s);
    if (tsq <= rms_sq) return T(kPi) * ssq;
    const T d = sqrt(tsq);
    const T ar = (tsq + rsq - ssq) / (T(2) * d);
    const T hsq = fmax(T(0.5) * (rsq + ssq) - (tsq * tsq + rps_sq * rms_sq) / (T(4) * tsq), T(0));
    const T h = sqrt(hsq);
    return rsq * atan2(h, ar) + ssq * atan2(h, d - ar) - d * h;
}

template <typename T>
__device__ inline T airy_kvalue(T t, T obs, T obssq)
{
    if constexpr (sizeof(T) == 4) {
        if (obs == T(0)) return airy_lens_same_f32<T>(T(1), t);
        return airy_lens_same_f32<T>(T(1), t) - T(2) * airy_lens_two_f32<T>(T(1), obs, T(1), obssq, t) +
               airy_lens_same_f32<T>(obssq, t);
    }
    if (obs == T(0)) {
        if (t >= T(4)) return T(0);
        if (t == T(0)) return T(kPi);
        const T hsq = fmax(T(1) - t / T(4), T(0));
        const T h = sqrt(hsq);
        return T(2) * (asin(fmin(h, T(1))) - h * sqrt(fmax(T(1) - hsq, T(0))));
    }
    return airy_circle_same<T>(T(1), T(1), t) - T(2) * airy_circle_two<T>(T(1), obs, T(1), obssq, t) +
           airy_circle_same<T>(obs, obssq, t);
}

// Device-side Ogata node tables (built once per device by gsb_init).
struct OgataTables {
    int lev_min, lev_max;            // h = 2^-lev for lev in [lev_min, lev_max]
    long long off[32];               // node offset of each level (index lev - lev_min)
    long long cnt[32];               // node count of each level
    const double2* xw;               // (log x, w) per node
    const double2* root;             // (j0 zero, Y0(z)/J1(z)) for s = 1..nroot
    long long nroot;
};

// One InterpolatedImage slot on the device: the caller's gsb_image_desc plus where its
// k-image (N rows q = 0..N-1 of N/2 + 1 columns p = 0..N/2) and row scratch live.
struct ImageSlot {
    gsb_image_desc desc;
    long long k_offset;      // element offset in d_k64 / d_k32
    long long row_offset;    // element offset in d_krows (ny rows of N/2 + 1)
};

// Library state per device.
struct DeviceState {
    bool ready = false;
    int sm_count = 0;
    double2* d_xw = nullptr;
    double2* d_root = nullptr;
    int* d_status = nullptr;      // status word of gsb_prepare_leaves
    OgataTables og{};
    // Kolmogorov stepk factors cached per GSParams key
    double kolm_key[13] = {0};
    double kolm_stepk = 0.;
    bool kolm_valid = false;
};

DeviceState* device_state();

}  // namespace gsb

// Opaque table set (device memory owned by the library).
struct gsb_tables {
    int count = 0;
    int stride = 0;               // nodes per slot
    double* d_header = nullptr;   // count * kSersicHeader
    double4* d_node = nullptr;    // count * stride
    double* d_val = nullptr;      // scratch: count * stride Hankel values
    void* d_scan = nullptr;       // scratch: per-slot state of the table's stopping scan
    double* d_n = nullptr;        // Sersic indices of the slots
    double* d_trunc = nullptr;    // truncation radius / r0 of the slots (when any is truncated)
    size_t cap_trunc = 0;
    int* d_status = nullptr;      // convergence status word
    size_t cap_slots = 0, cap_nodes = 0;
    // n-derivative tables (built on request)
    bool has_dn = false;
    double* d_dheader = nullptr;  // count * kSersicDHeader
    double4* d_dnode = nullptr;   // count * stride
    double* d_dval = nullptr;     // scratch: count * stride d/dn Hankel values
    size_t cap_dn_slots = 0, cap_dn_nodes = 0;
    // the device part of the last Sersic build as a CUDA graph, and what it was captured for
    cudaGraphExec_t sersic_exec = nullptr;
    unsigned char sersic_key[256] = {};
    cudaStream_t capture_stream = nullptr;
    // truncated Moffat slots (gsb_moffat_tables_build)
    int moffat_count = 0;
    int moffat_stride = 0;            // nodes per slot
    double* d_mheader = nullptr;      // moffat_count * kMoffatHeader
    double4* d_mnode = nullptr;       // moffat_count * moffat_stride
    double* d_mval = nullptr;         // scratch: Hankel values
    double* d_mk = nullptr;           // the k grid (moffat_stride)
    int* d_mstatus = nullptr;
    size_t cap_mslots = 0, cap_mnodes = 0, cap_mk = 0;
    // InterpolatedImage slots (gsb_images_build)
    int n_images = 0;
    gsb::ImageSlot* d_images = nullptr;   // n_images slot headers
    double* d_image_info = nullptr;       // n_images * 2: (R, maxk) in image units
    double2* d_k64 = nullptr;             // half-plane k-images, FP64
    float2* d_k32 = nullptr;              // the same, FP32
    double2* d_krows = nullptr;           // scratch: row transforms
    size_t cap_images = 0, cap_k = 0, cap_krows = 0;
};
