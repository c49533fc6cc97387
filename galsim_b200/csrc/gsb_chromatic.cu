// Wavelength integration of chromatic drawing: the weighted sum of a batch of monochromatic
// stamps of one geometry into one image,
//     out[p] = sum_s w[s] * stamp_s[p],
// the reference's IntegrationRule.__call__ (galsim/integ.py:134-146: sum(g * f(x) for g, x in
// zip(gs, xs)) over the images drawn at the integration wavelengths).  FP64 accumulation; each
// thread owns pixels p, p + stride, ... and reads stamp s's pixel p, so a warp's loads of one
// stamp are one coalesced segment.  HBM-bound: (n_stamps + 1) * npix elements move per call.
#include "gsb_internal.cuh"

namespace gsb {
namespace {

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256) weighted_stamp_sum_kernel(const Tin* __restrict__ flat,
                                                                 const long long* __restrict__ offsets,
                                                                 const double* __restrict__ w, int n,
                                                                 long long npix, Tout* __restrict__ out)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += stride) {
        double acc = 0.;
        for (int s = 0; s < n; ++s) acc += w[s] * (double)flat[offsets[s] + p];
        out[p] = (Tout)acc;
    }
}

template <typename Tin>
int launch_sum(const Tin* flat, const long long* offsets, const double* w, int n, long long npix, void* out,
               int out_dtype, cudaStream_t stream)
{
    const int sms = device_state()->sm_count > 0 ? device_state()->sm_count : 148;
    long long blocks = (npix + 255) / 256;
    if (blocks > 8LL * sms) blocks = 8LL * sms;
    if (out_dtype == GSB_F64)
        weighted_stamp_sum_kernel<Tin, double><<<(unsigned)blocks, 256, 0, stream>>>(flat, offsets, w, n, npix,
                                                                                    static_cast<double*>(out));
    else
        weighted_stamp_sum_kernel<Tin, float><<<(unsigned)blocks, 256, 0, stream>>>(flat, offsets, w, n, npix,
                                                                                   static_cast<float*>(out));
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

}  // namespace
}  // namespace gsb

extern "C" int gsb_weighted_stamp_sum(const void* d_flat, int in_dtype, const int64_t* d_offsets,
                                      const double* d_weights, int n_stamps, int64_t npix, void* d_out,
                                      int out_dtype, void* stream)
{
    using namespace gsb;
    if (n_stamps < 0 || npix < 0) return set_error(GSB_ERR_INVALID, "negative stamp count or size");
    if ((in_dtype != GSB_F32 && in_dtype != GSB_F64) || (out_dtype != GSB_F32 && out_dtype != GSB_F64))
        return set_error(GSB_ERR_INVALID, "dtypes must be GSB_F32 or GSB_F64");
    if (npix == 0) return GSB_OK;
    if (!d_out || (n_stamps > 0 && (!d_flat || !d_offsets || !d_weights)))
        return set_error(GSB_ERR_INVALID, "null argument");
    const cudaStream_t st = (cudaStream_t)stream;
    const long long* offs = reinterpret_cast<const long long*>(d_offsets);
    if (in_dtype == GSB_F64)
        return launch_sum(static_cast<const double*>(d_flat), offs, d_weights, n_stamps, npix, d_out, out_dtype, st);
    return launch_sum(static_cast<const float*>(d_flat), offs, d_weights, n_stamps, npix, d_out, out_dtype, st);
}
