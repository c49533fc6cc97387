// Adjoint entry points: dispatch to the per-size instantiations of adjoint_fused_kernel.
#include "gsb_adjoint.cuh"

namespace gsb {

#define GSB_ADJ_GROUP(name)                                                                       \
    int adjoint_launch_##name(int N, const AdjArgs& args, size_t work_bytes, cudaStream_t stream,  \
                              bool* handled);                                                      \
    bool adjoint_workspace_##name(int N, int n_stamps, size_t* bytes);
GSB_ADJ_GROUP(f32_small)
GSB_ADJ_GROUP(f32_large)
GSB_ADJ_GROUP(f64_small)
GSB_ADJ_GROUP(f64_large)
#undef GSB_ADJ_GROUP

static int adjoint_launch_f32(int N, const AdjArgs& args, size_t work_bytes, cudaStream_t stream, bool* handled)
{
    const int rc = adjoint_launch_f32_small(N, args, work_bytes, stream, handled);
    return *handled ? rc : adjoint_launch_f32_large(N, args, work_bytes, stream, handled);
}

static int adjoint_launch_f64(int N, const AdjArgs& args, size_t work_bytes, cudaStream_t stream, bool* handled)
{
    const int rc = adjoint_launch_f64_small(N, args, work_bytes, stream, handled);
    return *handled ? rc : adjoint_launch_f64_large(N, args, work_bytes, stream, handled);
}

static bool adjoint_workspace_f32(int N, int n_stamps, size_t* bytes)
{
    return adjoint_workspace_f32_small(N, n_stamps, bytes) || adjoint_workspace_f32_large(N, n_stamps, bytes);
}

static bool adjoint_workspace_f64(int N, int n_stamps, size_t* bytes)
{
    return adjoint_workspace_f64_small(N, n_stamps, bytes) || adjoint_workspace_f64_large(N, n_stamps, bytes);
}

bool is_large_fft(int N);
size_t adjoint_large_workspace_size(int N, int n_stamps, int precision);
int adjoint_large(const AdjArgs& args, int N, int precision, size_t work_bytes, cudaStream_t stream);

int adjoint_grad_count(const gsb_template* tpl) { return grad_count(*tpl); }

size_t adjoint_workspace_size(int N, int n_stamps, int precision)
{
    size_t b = 0;
    if (precision == GSB_F64 ? adjoint_workspace_f64(N, n_stamps, &b) : adjoint_workspace_f32(N, n_stamps, &b))
        return b;
    if (is_large_fft(N)) return adjoint_large_workspace_size(N, n_stamps, precision);
    return 0;
}

int adjoint_images(const gsb_template* tpl, int n_stamps, const gsb_leaf* d_leaves,
                   const gsb_phase* d_phases, const double* d_scales, const gsb_stamp* d_stamps,
                   const gsb_tables* t, int N, const void* d_cot, int cot_dtype, double* d_grad,
                   unsigned want, int precision, void* d_work, size_t work_bytes, cudaStream_t stream)
{
    bool sersic = false;
    for (int l = 0; l < tpl->n_leaves; ++l) sersic |= tpl->leaf_type[l] == GSB_SERSIC && ((want >> l) & 1u);
    if (sersic && (!t || !t->has_dn))
        return set_error(GSB_ERR_INVALID, "the adjoint of Sersic leaves needs tables built with n-derivatives");
    AdjArgs args;
    args.tpl = *tpl;
    args.n_stamps = n_stamps;
    args.leaves = d_leaves;
    args.phases = d_phases;
    args.scales = d_scales;
    args.stamps = d_stamps;
    args.sersic_header = t ? t->d_header : nullptr;
    args.sersic_node = t ? t->d_node : nullptr;
    args.sersic_dheader = (t && t->has_dn) ? t->d_dheader : nullptr;
    args.sersic_dnode = (t && t->has_dn) ? t->d_dnode : nullptr;
    args.sersic_stride = t ? t->stride : 0;
    args.cot = d_cot;
    args.cot_dtype = cot_dtype;
    args.grad = d_grad;
    args.want = want;
    args.work = d_work;
    if (n_stamps <= 0) return GSB_OK;
    bool handled = false;
    const int rc = precision == GSB_F64 ? adjoint_launch_f64(N, args, work_bytes, stream, &handled)
                                        : adjoint_launch_f32(N, args, work_bytes, stream, &handled);
    if (handled) return rc;
    // N > 1024: the split row / column kernels of the large draw path, in reverse
    if (is_large_fft(N)) return adjoint_large(args, N, precision, work_bytes, stream);
    return set_error(GSB_ERR_UNSUPPORTED, "adjoint FFT size " + std::to_string(N) +
                                          " is not built (supported: 2^a or 3*2^a, 32..16384)");
}

}  // namespace gsb
