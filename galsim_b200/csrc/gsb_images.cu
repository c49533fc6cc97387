// InterpolatedImage sources: the k-image of each zero-padded image and its stepk / maxk.
//
// Reference: SBInterpolatedImage::checkK (rfft of the padded image, src/SBInterpolatedImage.cpp:
// 450-464 with rfft, src/Image.cpp:730-812), CalculateSizeContainingFlux (:1084-1110) and
// calculateMaxK (:1146-1213), called from InterpolatedImage._getStepK / _getMaxK
// (galsim/interpolatedimage.py:647-685).
//
// The transform is a direct two-pass DFT over the image's nonzero region only (the padding is
// zero, so a 32 x 32 image in a 128 x 128 frame costs 32 rows and 32 terms per output rather
// than full-frame FFTs):
//   rows:  R(p, y) = sum_x I(x, y) tw[(p X) mod N],   p = 0..N/2, y over the region's rows
//   cols:  K(p, q) = sum_y R(p, y) tw[(q Y) mod N],   q = 0..N-1, stored p-major
// with tw[m] = exp(-2 pi i m / N) in shared memory and exact integer phase indices; FP64
// throughout, with an FP32 copy of K for FP32 draws.
#include <algorithm>
#include <vector>

#include "gsb_interp.cuh"
#include "gsb_internal.cuh"

namespace gsb {
namespace {

__device__ inline void fill_fwd_twiddles(double2* tw, int N)
{
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double s, c;
        sincospi(-2. * double(m) / double(N), &s, &c);
        tw[m] = make_double2(c, s);
    }
}

__device__ inline int pmod_int(long long a, int n)
{
    long long r = a % n;
    return int(r < 0 ? r + n : r);
}

// Pass 1: R(p, y) for every row of the nonzero region.  grid = (blocks, images).
__global__ void kimage_rows_kernel(const ImageSlot* slots, const double* pix, double2* rows)
{
    extern __shared__ double2 tw_rows[];
    const gsb_image_desc& d = slots[blockIdx.y].desc;
    const int N = d.N, H = N / 2 + 1;
    fill_fwd_twiddles(tw_rows, N);
    __syncthreads();
    const double* img = pix + d.pix_offset;
    double2* out = rows + slots[blockIdx.y].row_offset;
    const long long total = (long long)d.ny * H;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        const int y = int(o / H), p = int(o % H);
        const double* row = img + (size_t)y * d.nx;
        int m = pmod_int((long long)p * d.x0, N);
        double re = 0., im = 0.;
        for (int x = 0; x < d.nx; ++x) {
            const double v = row[x];
            const double2 w = tw_rows[m];
            re = fma(v, w.x, re);
            im = fma(v, w.y, im);
            m += p;
            if (m >= N) m -= N;
        }
        out[o] = make_double2(re, im);
    }
}

// Pass 2: K(p, q) for the whole half plane, stored p-major (K[p N + q]): the drawing kernels
// read it with the lanes of a warp on consecutive rows, i.e. consecutive q at a shared p.
// grid = (blocks, images).
__global__ void kimage_cols_kernel(const ImageSlot* slots, const double2* rows, double2* k64, float2* k32)
{
    extern __shared__ double2 tw_cols[];
    const gsb_image_desc& d = slots[blockIdx.y].desc;
    const int N = d.N, H = N / 2 + 1;
    fill_fwd_twiddles(tw_cols, N);
    __syncthreads();
    const double2* R = rows + slots[blockIdx.y].row_offset;
    double2* K = k64 + slots[blockIdx.y].k_offset;
    float2* K32 = k32 + slots[blockIdx.y].k_offset;
    const long long total = (long long)N * H;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        const int p = int(o / N), q = int(o % N);
        int m = pmod_int((long long)q * d.y0, N);
        double re = 0., im = 0.;
        for (int y = 0; y < d.ny; ++y) {
            const double2 r = R[(size_t)y * H + p];
            const double2 w = tw_cols[m];
            re = fma(r.x, w.x, fma(-r.y, w.y, re));
            im = fma(r.x, w.y, fma(r.y, w.x, im));
            m += q;
            if (m >= N) m -= N;
        }
        K[o] = make_double2(re, im);
        K32[o] = make_float2(float(re), float(im));
    }
}

// Pass 3: stepk radius and maxk of one image per block.
constexpr int kScanThreads = 256;

__global__ void __launch_bounds__(kScanThreads) kimage_scan_kernel(const ImageSlot* slots, const double* pix,
                                                                   const double2* k64, double maxk_threshold,
                                                                   double kacc, double* info)
{
    extern __shared__ double scan_smem[];
    const gsb_image_desc& d = slots[blockIdx.x].desc;
    const int N = d.N, H = N / 2 + 1, No2 = N / 2;
    const double* img = pix + d.pix_offset;
    // pixel at frame coordinates (X, Y); zero outside the region
    auto at = [&](int X, int Y) -> double {
        const int x = X - d.x0, y = Y - d.y0;
        if (x < 0 || x >= d.nx || y < 0 || y >= d.ny) return 0.;
        return img[(size_t)y * d.nx + x];
    };
    double R = 0., maxk = 0.;
    if (d.flags & GSB_IMAGE_STEPK) {
        // CalculateSizeContainingFlux: grow the centred box ring by ring until it holds the
        // target flux.  Each ring d (pixels with max(|X|, |Y|) = d) is summed by one thread in
        // the reference's order within the ring, then the rings are accumulated in order.
        double* ring = scan_smem;   // dmax + 1 entries
        const int dmax = min((d.bx1 - d.bx0) / 2, (d.by1 - d.by0) / 2);
        for (int r = 1 + threadIdx.x; r <= dmax; r += blockDim.x) {
            double s = 0.;
            for (int x = -r; x < r; ++x) {
                s += at(x, -r);
                s += at(r, x);
                s += at(-x, r);
                s += at(-r, -x);
            }
            ring[r] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const double sgn = d.stepk_target > 0. ? 1. : -1.;
            double flux = at(0, 0);
            int r = 1;
            for (; r <= dmax; ++r) {
                flux += ring[r];
                if (sgn * flux >= sgn * d.stepk_target) break;
            }
            R = r + 0.5;
        }
        __syncthreads();
    }
    if (d.flags & GSB_IMAGE_MAXK) {
        // calculateMaxK: the last square ring ix (in the kx >= 0 half plane) holding a value
        // with |K|^2 above the threshold, stopping after 5 rings in a row below it.  The ring
        // flags are found in parallel; the stopping rule then runs in order.
        unsigned char* above = reinterpret_cast<unsigned char*>(scan_smem);
        const double2* K = k64 + slots[blockIdx.x].k_offset;
        const double dk = kPi / No2;
        double thresh = maxk_threshold * d.flux;
        thresh *= thresh;
        const double max_maxk = d.maxk_limit > 0. ? d.maxk_limit
                                                  : (d.x_interp == GSB_INTERP_LANCZOS ? d.x_table[3]
                                                                                      : interp_urange(d.x_interp, kacc)) /
                                                        (1. / (2. * kPi));
        int max_ix = int(ceil(max_maxk / dk));
        if (max_ix > No2) max_ix = No2;
        for (int ix = threadIdx.x; ix <= max_ix; ix += blockDim.x) above[ix] = 0;
        __syncthreads();
        // kimage(p, q) with p in 0..No2, q in -No2..No2-1 (stored p-major)
        auto nrm = [&](int p, int q) -> double {
            const double2 v = K[(size_t)p * N + (q < 0 ? q + N : q)];
            return v.x * v.x + v.y * v.y;
        };
        for (int ix = 0; ix <= max_ix; ++ix) {
            for (int iy = threadIdx.x; iy <= ix; iy += blockDim.x) {
                bool hit = nrm(iy, -ix) > thresh;
                if (!hit && iy != ix && ix != No2) hit = nrm(iy, ix) > thresh;
                if (!hit && iy > 0) hit = nrm(ix, -iy) > thresh;
                if (!hit && ix > 0 && iy != No2) hit = nrm(ix, iy) > thresh;
                if (hit) above[ix] = 1;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int maxk_ix = 0, below = 0;
            for (int ix = 0; ix <= max_ix; ++ix) {
                if (above[ix]) { maxk_ix = ix; below = 0; }
                if (++below == 5) break;
            }
            maxk = double(maxk_ix + 1) * dk;
        }
    }
    if (threadIdx.x == 0) {
        info[2 * blockIdx.x] = R;
        info[2 * blockIdx.x + 1] = maxk;
    }
}

template <typename P>
int grow(P*& p, size_t& cap, size_t need)
{
    if (need <= cap && p) return GSB_OK;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    GSB_CUDA_CHECK(cudaMalloc(&p, sizeof(P) * need));
    cap = need;
    return GSB_OK;
}

}  // namespace

int images_build(gsb_tables* t, int count, const gsb_image_desc* h_desc, const double* d_pixels,
                 const gsb_gsparams* gsp, cudaStream_t stream)
{
    DeviceState* st = device_state();
    if (!st->ready) return set_error(GSB_ERR_INVALID, "gsb_init has not been called");
    std::vector<ImageSlot> slots(count);
    long long k_total = 0, row_total = 0;
    int maxN = 0, max_half = 0;
    for (int i = 0; i < count; ++i) {
        const gsb_image_desc& d = h_desc[i];
        const int h = d.N / 2;
        if (d.N < 2 || d.N % 2 || d.N > GSB_IMAGE_MAX_N)
            return set_error(GSB_ERR_INVALID, "image frame size must be even and at most " +
                                                  std::to_string(GSB_IMAGE_MAX_N));
        if (d.nx < 1 || d.ny < 1 || d.x0 < -h || d.y0 < -h || d.x0 + d.nx > h || d.y0 + d.ny > h)
            return set_error(GSB_ERR_INVALID, "image region does not fit its padded frame");
        if ((d.flags & GSB_IMAGE_STEPK) &&
            (d.bx0 > 0 || d.bx1 < 0 || d.by0 > 0 || d.by1 < 0 || d.bx0 < d.x0 || d.by0 < d.y0 ||
             d.bx1 >= d.x0 + d.nx || d.by1 >= d.y0 + d.ny))
            return set_error(GSB_ERR_INVALID, "stepk bounds must contain (0, 0) and lie in the region");
        if (d.x_interp < GSB_INTERP_DELTA || d.x_interp > GSB_INTERP_SINC)
            return set_error(GSB_ERR_INVALID, "unknown x interpolant");
        if ((d.x_interp == GSB_INTERP_LANCZOS) != (d.x_table != nullptr))
            return set_error(GSB_ERR_INVALID, "a Lanczos x interpolant needs its x_table (and only it)");
        if (d.pix_offset < 0) return set_error(GSB_ERR_INVALID, "negative pixel offset");
        slots[i].desc = d;
        slots[i].k_offset = k_total;
        slots[i].row_offset = row_total;
        k_total += (long long)d.N * (h + 1);
        row_total += (long long)d.ny * (h + 1);
        maxN = std::max(maxN, d.N);
        max_half = std::max(max_half, h + 1);
    }
    t->n_images = 0;
    if (count == 0) return GSB_OK;
    int rc;
    const size_t cap_info = t->cap_images;   // d_image_info follows the slot capacity
    if ((rc = grow(t->d_images, t->cap_images, (size_t)count))) return rc;
    if (cap_info != t->cap_images || !t->d_image_info) {
        cudaFree(t->d_image_info);
        t->d_image_info = nullptr;
        GSB_CUDA_CHECK(cudaMalloc(&t->d_image_info, sizeof(double) * 2 * t->cap_images));
    }
    const size_t cap_k32 = t->cap_k;           // d_k32 follows the d_k64 capacity
    if ((rc = grow(t->d_k64, t->cap_k, (size_t)k_total))) return rc;
    if (cap_k32 != t->cap_k || !t->d_k32) {
        cudaFree(t->d_k32);
        t->d_k32 = nullptr;
        GSB_CUDA_CHECK(cudaMalloc(&t->d_k32, sizeof(float2) * t->cap_k));
    }
    if ((rc = grow(t->d_krows, t->cap_krows, (size_t)row_total))) return rc;
    GSB_CUDA_CHECK(cudaMemcpyAsync(t->d_images, slots.data(), sizeof(ImageSlot) * count,
                                   cudaMemcpyHostToDevice, stream));

    const size_t tw_bytes = sizeof(double2) * maxN;
    if (tw_bytes > 48 * 1024) {
        GSB_CUDA_CHECK(cudaFuncSetAttribute(kimage_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)tw_bytes));
        GSB_CUDA_CHECK(cudaFuncSetAttribute(kimage_cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)tw_bytes));
    }
    // enough blocks per image to fill the SMs when there are few images
    const int per_image = std::max(1, std::min(64, 2 * st->sm_count / std::max(1, count)));
    kimage_rows_kernel<<<dim3(per_image, count), 256, tw_bytes, stream>>>(t->d_images, d_pixels, t->d_krows);
    GSB_CUDA_CHECK(cudaGetLastError());
    kimage_cols_kernel<<<dim3(per_image, count), 256, tw_bytes, stream>>>(t->d_images, t->d_krows, t->d_k64,
                                                                          t->d_k32);
    GSB_CUDA_CHECK(cudaGetLastError());
    const size_t scan_bytes = sizeof(double) * (max_half + 1);
    kimage_scan_kernel<<<count, kScanThreads, scan_bytes, stream>>>(t->d_images, d_pixels, t->d_k64,
                                                                    gsp->maxk_threshold, gsp->kvalue_accuracy,
                                                                    t->d_image_info);
    GSB_CUDA_CHECK(cudaGetLastError());
    // the slot headers are copied from host memory owned by this call
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    t->n_images = count;
    return GSB_OK;
}

}  // namespace gsb

using namespace gsb;

extern "C" int gsb_images_build(gsb_tables* t, int count, const gsb_image_desc* h_desc,
                                const double* d_pixels, const gsb_gsparams* gsp, void* stream)
{
    if (!t || !gsp || count < 0 || (count > 0 && (!h_desc || !d_pixels)))
        return set_error(GSB_ERR_INVALID, "null argument");
    return images_build(t, count, h_desc, d_pixels, gsp, (cudaStream_t)stream);
}

extern "C" int gsb_images_info(const gsb_tables* t, double* h_out, int count, void* stream)
{
    if (!t || (count > 0 && !h_out)) return set_error(GSB_ERR_INVALID, "null argument");
    if (count < 0 || count > t->n_images) return set_error(GSB_ERR_INVALID, "count exceeds built images");
    if (count == 0) return GSB_OK;
    GSB_CUDA_CHECK(cudaMemcpyAsync(h_out, t->d_image_info, sizeof(double) * 2 * count,
                                   cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return GSB_OK;
}
