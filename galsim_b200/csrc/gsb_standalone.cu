// The reference's four _galsim hot-path bindings as standalone entry points, for callers that
// keep the reference's own drawFFT orchestration (galsim/gsobject.py:2014-2045) and replace only
// the compiled steps it calls:
//   gsb_draw_k               SBProfile.drawK           pysrc/SBProfile.cpp:35-40, src/SBProfile.cpp:383-425
//   gsb_apply_kimage_phases  ApplyKImagePhases         pysrc/SBTransform.cpp:27-40, src/SBTransform.cpp:740-883
//   gsb_wrap_image           wrapImage                 pysrc/Image.cpp:60-61, src/Image.cpp:578-727
//   gsb_irfft                irfft                     pysrc/Image.cpp:53-57, src/Image.cpp:815-912
// Each works on one image in device memory.  The batched path (gsb_draw_images) fuses all four
// and never writes a k-image to HBM; these exist for the drop-in at the reference's boundary.
#include <algorithm>

#include "gsb_draw.cuh"

namespace gsb {

int draw_kimages(const gsb_template* tpl, int n_stamps, const gsb_leaf* d_leaves,
                 const gsb_phase* d_phases, const double* d_scales, const gsb_tables* t, double dk,
                 int kxmin, int kymin, int nkx, int nky, void* d_out, int out_dtype,
                 cudaStream_t stream);
int fft_twiddles(int N, cudaStream_t stream, const double2** out);

namespace {

struct Jac { double a, b, c, d; };

// jac1 = jac . J for every leaf and phase record (Transformation._drawKImage, transform.py:592:
// the caller's jac multiplies the records' own composed Jacobians from the left), with the
// general-Jacobian flags recomputed as the reference's fill chooses (off-diagonal terms != 0).
__global__ void compose_jac_kernel(const gsb_leaf* in_l, gsb_leaf* out_l, long long n_leaf,
                                   const gsb_phase* in_p, gsb_phase* out_p, long long n_phase, Jac J)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n_leaf) {
        gsb_leaf L = in_l[i];
        const double A = L.jac[0], B = L.jac[1], C = L.jac[2], D = L.jac[3];
        L.jac[0] = J.a * A + J.b * C;
        L.jac[1] = J.a * B + J.b * D;
        L.jac[2] = J.c * A + J.d * C;
        L.jac[3] = J.c * B + J.d * D;
        L.flags = (L.flags & ~GSB_LEAF_JAC_GENERAL) |
                  ((L.jac[1] != 0. || L.jac[2] != 0.) ? GSB_LEAF_JAC_GENERAL : 0);
        out_l[i] = L;
    }
    if (i < n_phase) {
        gsb_phase P = in_p[i];
        const double A = P.jac[0], B = P.jac[1], C = P.jac[2], D = P.jac[3];
        P.jac[0] = J.a * A + J.b * C;
        P.jac[1] = J.a * B + J.b * D;
        P.jac[2] = J.c * A + J.d * C;
        P.jac[3] = J.c * B + J.d * D;
        P.flags = (P.flags & ~GSB_PHASE_JAC_GENERAL) |
                  ((P.jac[1] != 0. || P.jac[2] != 0.) ? GSB_PHASE_JAC_GENERAL : 0);
        out_p[i] = P;
    }
}

// image(i, j) *= fs exp(-i (kx' cx + ky' cy)), kx = i dk, ky = j dk, (kx', ky') = (A kx + C ky,
// B kx + D ky); the phase in FP64 turns, reduced to [-1/2, 1/2] before sincospi.
template <typename T>
__global__ void apply_phases_kernel(Cx<T>* img, int nx, int ny, long long stride, int xmin, int ymin,
                                    double ax, double ay, double fs)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)nx * ny) return;
    const int c = int(idx % nx), r = int(idx / nx);
    double tt = double(xmin + c) * ax + double(ymin + r) * ay;
    tt -= rint(tt);
    double sn, cs;
    sincospi(-2. * tt, &sn, &cs);
    Cx<T>& v = img[(long long)r * stride + c];
    const double re = double(v.x), im = double(v.y);
    v.x = T(fs * (re * cs - im * sn));
    v.y = T(fs * (re * sn + im * cs));
}

// Every cell (x, y) of the target bounds gets the compensated sum of its aliases
// (x + a Px, y + b Py) in the input (Px, Py the target's widths).  hermx: the input holds
// x >= 0 only, with X(-x, -y) = conj X(x, y), and the x period is N = 2 (mwrap - 1): an alias
// at x' < 0 reads conj X(-x', -y').  This is the sum that the reference's in-place pointer walk
// forms; it is written to a separate output.
template <typename V, bool CPLX, bool HERMX>
__global__ void wrap_kernel(const V* in, int m, int n, long long in_stride, int in_xmin, int in_ymin,
                            V* out, long long out_stride, int bxmin, int bymin, int mwrap, int nwrap)
{
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)mwrap * nwrap) return;
    const int ox = int(idx % mwrap), oy = int(idx / mwrap);
    const int x = bxmin + ox, y = bymin + oy;
    const int px = HERMX ? 2 * (mwrap - 1) : mwrap;
    const int xlo = HERMX ? -(m - 1) : in_xmin, xhi = HERMX ? m - 1 : in_xmin + m - 1;
    const int ylo = in_ymin, yhi = in_ymin + n - 1;
    double sr = 0., si = 0., cr = 0., ci = 0.;       // Kahan sums
    auto add = [](double& s, double& c, double v) {
        const double yv = v - c, t = s + yv;
        c = (t - s) - yv;
        s = t;
    };
    for (int xp = x + px * ((xlo - x) / px - 1); xp <= xhi; xp += px) {
        if (xp < xlo) continue;
        for (int yp = y + nwrap * ((ylo - y) / nwrap - 1); yp <= yhi + nwrap; yp += nwrap) {
            const bool neg = HERMX && xp < 0;
            const int rx = neg ? -xp : xp, ry = neg ? -yp : yp;
            if (ry < ylo || ry > yhi) continue;
            const V v = in[(long long)(ry - in_ymin) * in_stride + (rx - (HERMX ? 0 : in_xmin))];
            if constexpr (CPLX) {
                add(sr, cr, double(v.x));
                add(si, ci, neg ? -double(v.y) : double(v.y));
            } else {
                add(sr, cr, double(v));
            }
        }
    }
    V o;
    if constexpr (CPLX) { o.x = decltype(o.x)(sr); o.y = decltype(o.y)(si); }
    else o = V(sr);
    out[(long long)oy * out_stride + ox] = o;
}

// irfft, first pass: column c (kx = c) of the half plane, its Ny values taken in FFTW's row
// order (shift_in: ky = 0 .. Ny/2-1 first, then -Ny/2 .. -1) and scaled by 1/(Nx Ny) and, with
// shift_out, by (-1)^(c + row); then the inverse DFT along y.  The imaginary parts of the
// kx = 0 and kx = Nx/2 columns are dropped after it, as a c2r transform does.
template <typename T>
__global__ void __launch_bounds__(1024) irfft_col_kernel(const Cx<T>* in, long long in_stride, int Nx, int Ny, int shift_in,
                                 int shift_out, const double2* tw, double2* W)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* buf = reinterpret_cast<double2*>(sm_raw);
    const int H = Nx / 2 + 1;
    const double fac = 1. / (double(Nx) * double(Ny));
    for (int c = blockIdx.x; c < H; c += gridDim.x) {
        for (int r = threadIdx.x; r < Ny; r += blockDim.x) {
            // FFTW row r holds ky = r (r < Ny/2) else r - Ny; input row index is ky + Ny/2
            const int ky = r < Ny / 2 ? r : r - Ny;
            const int src = shift_in ? ky + Ny / 2 : r;
            const Cx<T> v = in[(long long)src * in_stride + c];
            const double f = (shift_out && ((c + r) & 1)) ? -fac : fac;
            buf[r] = make_double2(f * double(v.x), f * double(v.y));
        }
        __syncthreads();
        block_fft<double, +1>(buf, Ny, tw);
        for (int r = threadIdx.x; r < Ny; r += blockDim.x) {
            double2 v = buf[r];
            if (c == 0 || c == H - 1) v.y = 0.;
            W[(long long)c * Ny + r] = v;
        }
        __syncthreads();
    }
}

// irfft, second pass: two output rows per transform (row1 + i row2, each Hermitian-extended in
// kx), the inverse DFT along x; real parts to out rows of Nx + 2 doubles (the reference's
// output bounds -Nx/2 .. Nx/2+1; the last two columns are left as they are).
__global__ void __launch_bounds__(1024) irfft_row_kernel(const double2* W, int Nx, int Ny, const double2* tw, double* out,
                                 long long out_stride)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double2* buf = reinterpret_cast<double2*>(sm_raw);
    const int H = Nx / 2 + 1;
    for (int p = blockIdx.x; p < Ny / 2; p += gridDim.x) {
        const int y1 = 2 * p, y2 = 2 * p + 1;
        for (int kx = threadIdx.x; kx < Nx; kx += blockDim.x) {
            double2 a1, a2;
            if (kx < H) {
                a1 = W[(long long)kx * Ny + y1];
                a2 = W[(long long)kx * Ny + y2];
            } else {
                a1 = W[(long long)(Nx - kx) * Ny + y1];
                a2 = W[(long long)(Nx - kx) * Ny + y2];
                a1.y = -a1.y;
                a2.y = -a2.y;
            }
            buf[kx] = make_double2(a1.x - a2.y, a1.y + a2.x);
        }
        __syncthreads();
        block_fft<double, +1>(buf, Nx, tw);
        for (int x = threadIdx.x; x < Nx; x += blockDim.x) {
            out[(long long)y1 * out_stride + x] = buf[x].x;
            out[(long long)y2 * out_stride + x] = buf[x].y;
        }
        __syncthreads();
    }
}

int block_threads(int N)
{
    // one thread per butterfly of a radix-2 pass at least, 128 .. 1024
    int t = 128;
    while (t < N / 2 && t < 1024) t *= 2;
    return t;
}

}  // namespace

}  // namespace gsb

using namespace gsb;

extern "C" {

int gsb_draw_k(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp, const gsb_leaf* d_leaves,
               const gsb_phase* d_phases, const double* d_scales, const gsb_tables* t, double dk,
               const double* jac, int xmin, int ymin, int nx, int ny, void* d_out, int out_dtype,
               void* stream)
{
    int rc = validate_template(tpl);
    if (rc) return rc;
    if (!gsp) return set_error(GSB_ERR_INVALID, "null gsparams");
    if (n_stamps < 0 || nx < 0 || ny < 0) return set_error(GSB_ERR_INVALID, "negative size");
    if (n_stamps == 0 || nx == 0 || ny == 0) return GSB_OK;
    if (!d_leaves || !d_out || (tpl->n_phases && !d_phases) || (tpl->n_scales && !d_scales))
        return set_error(GSB_ERR_INVALID, "null device pointer");
    if (out_dtype != GSB_F32 && out_dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad out_dtype");
    if (!(dk > 0.)) return set_error(GSB_ERR_INVALID, "dk must be > 0");
    cudaStream_t s = (cudaStream_t)stream;
    if (!jac)
        return draw_kimages(tpl, n_stamps, d_leaves, d_phases, d_scales, t, dk, xmin, ymin, nx, ny, d_out,
                            out_dtype, s);
    const long long nl = (long long)n_stamps * tpl->n_leaves, np = (long long)n_stamps * tpl->n_phases;
    gsb_leaf* l2 = nullptr;
    gsb_phase* p2 = nullptr;
    GSB_CUDA_CHECK(cudaMallocAsync(&l2, sizeof(gsb_leaf) * nl, s));
    if (np) {
        const cudaError_t e = cudaMallocAsync(&p2, sizeof(gsb_phase) * np, s);
        if (e != cudaSuccess) {
            cudaFreeAsync(l2, s);
            return set_error(GSB_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
        }
    }
    const long long nmax = std::max(nl, np);
    compose_jac_kernel<<<(unsigned)((nmax + 255) / 256), 256, 0, s>>>(d_leaves, l2, nl, d_phases, p2, np,
                                                                       Jac{jac[0], jac[1], jac[2], jac[3]});
    rc = cudaGetLastError() == cudaSuccess ? GSB_OK : set_error(GSB_ERR_CUDA, "compose_jac_kernel launch");
    if (rc == GSB_OK)
        rc = draw_kimages(tpl, n_stamps, l2, p2, d_scales, t, dk, xmin, ymin, nx, ny, d_out, out_dtype, s);
    cudaFreeAsync(l2, s);
    if (p2) cudaFreeAsync(p2, s);
    return rc;
}

int gsb_apply_kimage_phases(void* d_image, int dtype, int xmin, int ymin, int nx, int ny, long long stride,
                            double dk, const double* jac, double cenx, double ceny, double flux_scaling,
                            void* stream)
{
    if (nx < 0 || ny < 0 || stride < nx) return set_error(GSB_ERR_INVALID, "bad image size or stride");
    if (nx == 0 || ny == 0) return GSB_OK;
    if (!d_image) return set_error(GSB_ERR_INVALID, "null device pointer");
    if (dtype != GSB_F32 && dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad dtype");
    const double A = jac ? jac[0] : 1., B = jac ? jac[1] : 0., C = jac ? jac[2] : 0., D = jac ? jac[3] : 1.;
    // kx' cx + ky' cy = kx (A cx + B cy) + ky (C cx + D cy), in turns of 2 pi
    const double ax = dk * (A * cenx + B * ceny) / (2. * kPi);
    const double ay = dk * (C * cenx + D * ceny) / (2. * kPi);
    const long long n = (long long)nx * ny;
    const unsigned g = (unsigned)((n + 255) / 256);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == GSB_F64)
        apply_phases_kernel<double><<<g, 256, 0, s>>>(static_cast<Cx<double>*>(d_image), nx, ny, stride, xmin,
                                                      ymin, ax, ay, flux_scaling);
    else
        apply_phases_kernel<float><<<g, 256, 0, s>>>(static_cast<Cx<float>*>(d_image), nx, ny, stride, xmin,
                                                     ymin, ax, ay, flux_scaling);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

int gsb_wrap_image(const void* d_in, int dtype, int is_complex, int xmin, int xmax, int ymin, int ymax,
                   long long in_stride, int bxmin, int bxmax, int bymin, int bymax, int hermx, int hermy,
                   void* d_out, long long out_stride, void* stream)
{
    const int m = xmax - xmin + 1, n = ymax - ymin + 1;
    const int mwrap = bxmax - bxmin + 1, nwrap = bymax - bymin + 1;
    if (m <= 0 || n <= 0 || mwrap <= 0 || nwrap <= 0) return set_error(GSB_ERR_INVALID, "undefined bounds");
    if (bxmin < xmin || bxmax > xmax || bymin < ymin || bymax > ymax)
        return set_error(GSB_ERR_INVALID, "wrap bounds must lie inside the image bounds");
    if (in_stride < m || out_stride < mwrap) return set_error(GSB_ERR_INVALID, "bad stride");
    if (!d_in || !d_out) return set_error(GSB_ERR_INVALID, "null device pointer");
    if (dtype != GSB_F32 && dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad dtype");
    if (hermy) return set_error(GSB_ERR_UNSUPPORTED, "wrapImage with hermy is not built (drawFFT wraps "
                                                     "with hermx)");
    if (hermx) {
        // image.py:766-782: xmin == 0 in both, y symmetric in the image, the wrap bounds missing
        // their most negative row
        if (!is_complex) return set_error(GSB_ERR_INVALID, "hermx needs a complex image");
        if (xmin != 0 || bxmin != 0)
            return set_error(GSB_ERR_INVALID, "hermitian == 'x' requires xmin == 0 and bounds.xmin == 0");
        if (ymin != -ymax || bymin != -bymax - 1)
            return set_error(GSB_ERR_INVALID, "hermitian == 'x' requires symmetric y bounds");
    }
    const long long cells = (long long)mwrap * nwrap;
    const unsigned g = (unsigned)((cells + 255) / 256);
    cudaStream_t s = (cudaStream_t)stream;
#define GSB_WRAP(V, C, H)                                                                         \
    wrap_kernel<V, C, H><<<g, 256, 0, s>>>(static_cast<const V*>(d_in), m, n, in_stride, xmin, ymin, \
                                           static_cast<V*>(d_out), out_stride, bxmin, bymin, mwrap, nwrap)
    if (is_complex) {
        if (dtype == GSB_F64) { if (hermx) GSB_WRAP(double2, true, true); else GSB_WRAP(double2, true, false); }
        else { if (hermx) GSB_WRAP(float2, true, true); else GSB_WRAP(float2, true, false); }
    } else {
        if (dtype == GSB_F64) GSB_WRAP(double, false, false);
        else GSB_WRAP(float, false, false);
    }
#undef GSB_WRAP
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

int gsb_irfft(const void* d_in, int in_dtype, int Nx, int Ny, long long in_stride, double* d_out,
              long long out_stride, int shift_in, int shift_out, void* d_work, size_t work_bytes,
              void* stream)
{
    if (Nx < 2 || Ny < 2 || (Nx & 1) || (Ny & 1)) return set_error(GSB_ERR_INVALID, "Nx, Ny must be even and >= 2");
    if (!good_fft_size_ok(Nx) || !good_fft_size_ok(Ny))
        return set_error(GSB_ERR_UNSUPPORTED, "irfft sizes other than 2^a or 3*2^a are not built");
    // one FP64 column or row in shared memory: 16 B x N <= 227 KB
    if (Nx > 12288 || Ny > 12288) return set_error(GSB_ERR_UNSUPPORTED, "irfft sizes above 12288 are not built");
    if (in_stride < Nx / 2 + 1 || out_stride < Nx + 2) return set_error(GSB_ERR_INVALID, "bad stride");
    if (!d_in || !d_out || !d_work) return set_error(GSB_ERR_INVALID, "null device pointer");
    if (in_dtype != GSB_F32 && in_dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad dtype");
    if (work_bytes < sizeof(double2) * (size_t)(Nx / 2 + 1) * Ny)
        return set_error(GSB_ERR_INVALID, "irfft workspace too small (gsb_irfft_workspace_size)");
    cudaStream_t s = (cudaStream_t)stream;
    const double2 *twx = nullptr, *twy = nullptr;
    int rc = fft_twiddles(Nx, s, &twx);
    if (rc) return rc;
    rc = fft_twiddles(Ny, s, &twy);
    if (rc) return rc;
    double2* W = static_cast<double2*>(d_work);
    const int tc = block_threads(Ny), tr = block_threads(Nx);
    const size_t smc = sizeof(double2) * Ny, smr = sizeof(double2) * Nx;
    if (smc > 48 * 1024)
        GSB_CUDA_CHECK(cudaFuncSetAttribute(in_dtype == GSB_F64 ? (const void*)irfft_col_kernel<double>
                                                                : (const void*)irfft_col_kernel<float>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(smc)));
    if (smr > 48 * 1024)
        GSB_CUDA_CHECK(cudaFuncSetAttribute((const void*)irfft_row_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(smr)));
    const int H = Nx / 2 + 1;
    if (in_dtype == GSB_F64)
        irfft_col_kernel<double><<<std::min(H, 1184), tc, smc, s>>>(static_cast<const Cx<double>*>(d_in), in_stride,
                                                                    Nx, Ny, shift_in, shift_out, twy, W);
    else
        irfft_col_kernel<float><<<std::min(H, 1184), tc, smc, s>>>(static_cast<const Cx<float>*>(d_in), in_stride,
                                                                   Nx, Ny, shift_in, shift_out, twy, W);
    GSB_CUDA_CHECK(cudaGetLastError());
    irfft_row_kernel<<<std::min(Ny / 2, 1184), tr, smr, s>>>(W, Nx, Ny, twx, d_out, out_stride);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

size_t gsb_irfft_workspace_size(int Nx, int Ny)
{
    if (Nx < 2 || Ny < 2) return 0;
    return sizeof(double2) * (size_t)(Nx / 2 + 1) * Ny;
}

}  // extern "C"
