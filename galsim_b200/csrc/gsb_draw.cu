// Public draw entry points: dispatch to the per-size kernel instantiations.
#include "gsb_draw.cuh"

namespace gsb {

#define GSB_GROUP(name)                                                                        \
    int fused_launch_##name(int N, const DrawArgs& args, size_t work_bytes, cudaStream_t stream, \
                            bool* handled);                                                    \
    bool fused_workspace_##name(int N, int n_stamps, size_t* bytes);
GSB_GROUP(f32_small)
GSB_GROUP(f32_large)
GSB_GROUP(f64_small)
GSB_GROUP(f64_large)
#undef GSB_GROUP

bool is_large_fft(int N);
size_t large_workspace_size(int N, int n_stamps, int precision);
int draw_large(const DrawArgs& args, int N, int precision, void* work, size_t work_bytes,
               cudaStream_t stream);

size_t draw_workspace_size(int N, int n_stamps, int precision)
{
    if (is_large_fft(N)) return large_workspace_size(N, n_stamps, precision);
    size_t b = 0;
    if (precision == GSB_F64) {
        if (fused_workspace_f64_small(N, n_stamps, &b) || fused_workspace_f64_large(N, n_stamps, &b)) return b;
    } else {
        if (fused_workspace_f32_small(N, n_stamps, &b) || fused_workspace_f32_large(N, n_stamps, &b)) return b;
    }
    return 0;
}

int draw_images(const gsb_template* tpl, int n_stamps, const gsb_leaf* d_leaves,
                const gsb_phase* d_phases, const double* d_scales, const gsb_stamp* d_stamps,
                const gsb_tables* t, int N, void* d_out, int out_dtype, int add,
                double* d_added_flux, int precision, void* d_work, size_t work_bytes,
                cudaStream_t stream)
{
    DrawArgs args;
    args.tpl = *tpl;
    args.n_stamps = n_stamps;
    args.leaves = d_leaves;
    args.phases = d_phases;
    args.scales = d_scales;
    args.stamps = d_stamps;
    args.sersic_header = t ? t->d_header : nullptr;
    args.sersic_node = t ? t->d_node : nullptr;
    args.sersic_stride = t ? t->stride : 0;
    args.out = d_out;
    args.out_dtype = out_dtype;
    args.add = add;
    args.added_flux = d_added_flux;
    args.work = d_work;
    if (n_stamps <= 0) return GSB_OK;
    if (is_large_fft(N)) return draw_large(args, N, precision, d_work, work_bytes, stream);
    bool handled = false;
    int rc;
    if (precision == GSB_F64) {
        rc = fused_launch_f64_small(N, args, work_bytes, stream, &handled);
        if (!handled) rc = fused_launch_f64_large(N, args, work_bytes, stream, &handled);
    } else {
        rc = fused_launch_f32_small(N, args, work_bytes, stream, &handled);
        if (!handled) rc = fused_launch_f32_large(N, args, work_bytes, stream, &handled);
    }
    if (!handled)
        return set_error(GSB_ERR_UNSUPPORTED, "FFT size " + std::to_string(N) +
                                              " is not built (supported: 2^a or 3*2^a, 32..16384)");
    return rc;
}

int draw_kimages(const gsb_template* tpl, int n_stamps, const gsb_leaf* d_leaves,
                 const gsb_phase* d_phases, const double* d_scales, const gsb_tables* t, double dk,
                 int kxmin, int kymin, int nkx, int nky, void* d_out, int out_dtype,
                 cudaStream_t stream)
{
    if (n_stamps <= 0 || nkx <= 0 || nky <= 0) return GSB_OK;
    const long long per = (long long)nkx * nky;
    dim3 grid((unsigned)std::min<long long>((per + 255) / 256, 1024), (unsigned)std::min(n_stamps, 65535));
    const double* sh = t ? t->d_header : nullptr;
    const double4* sn = t ? t->d_node : nullptr;
    const int ss = t ? t->stride : 0;
    if (out_dtype == GSB_F64)
        draw_kimage_kernel<double><<<grid, 256, 0, stream>>>(*tpl, n_stamps, d_leaves, d_phases, d_scales,
                                                             sh, sn, ss, dk, kxmin, kymin, nkx, nky,
                                                             d_out, out_dtype);
    else
        draw_kimage_kernel<float><<<grid, 256, 0, stream>>>(*tpl, n_stamps, d_leaves, d_phases, d_scales,
                                                            sh, sn, ss, dk, kxmin, kymin, nkx, nky,
                                                            d_out, out_dtype);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

}  // namespace gsb
