// extern "C" entry points of libgsb.so (declared in include/gsb.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "gsb_internal.cuh"

namespace gsb {

int ogata_init(DeviceState* st);
int sersic_truncation(int count, const double* h_in, double* h_out, cudaStream_t stream);
int moffat_tables_build(gsb_tables* t, const double* h_beta, const double* h_trunc, int count,
                        const gsb_gsparams* gsp, cudaStream_t stream);
int moffat_scale_radius(int count, const double* h_in, double* h_out, cudaStream_t stream);
int sersic_tables_build(gsb_tables* t, const double* h_n, const double* h_trunc, int count,
                        const gsb_gsparams* gsp, bool with_dn, cudaStream_t stream);
int adjoint_grad_count(const gsb_template* tpl);
size_t adjoint_workspace_size(int N, int n_stamps, int precision);
int adjoint_images(const gsb_template* tpl, int n_stamps, const gsb_leaf* d_leaves,
                   const gsb_phase* d_phases, const double* d_scales, const gsb_stamp* d_stamps,
                   const gsb_tables* t, int N, const void* d_cot, int cot_dtype, double* d_grad,
                   unsigned want, int precision, void* d_work, size_t work_bytes, cudaStream_t stream);
int prepare_leaves(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp, gsb_leaf* d_leaves,
                   const gsb_tables* t, double* d_info, cudaStream_t stream);
size_t draw_workspace_size(int N, int n_stamps, int precision);
int draw_set_variant(int v);
int exp_fp64(const double* d_x, double* d_y, int n, int table_size, cudaStream_t stream);
int draw_tune_report(char* buf, size_t len);
int draw_images(const gsb_template* tpl, int n_stamps, const gsb_leaf* d_leaves,
                const gsb_phase* d_phases, const double* d_scales, const gsb_stamp* d_stamps,
                const gsb_tables* t, int N, void* d_out, int out_dtype, int add,
                double* d_added_flux, int precision, void* d_work, size_t work_bytes,
                cudaStream_t stream);
int draw_kimages(const gsb_template* tpl, int n_stamps, const gsb_leaf* d_leaves,
                 const gsb_phase* d_phases, const double* d_scales, const gsb_tables* t, double dk,
                 int kxmin, int kymin, int nkx, int nky, void* d_out, int out_dtype,
                 cudaStream_t stream);

namespace {
thread_local std::string g_err;
std::mutex g_mu;
DeviceState g_state[64];
}  // namespace

int validate_template(const gsb_template* tpl)
{
    if (!tpl) return set_error(GSB_ERR_INVALID, "null template");
    if (tpl->n_ops < 1 || tpl->n_ops > GSB_MAX_OPS || tpl->n_leaves < 1 ||
        tpl->n_leaves > GSB_MAX_LEAVES || tpl->n_phases < 0 || tpl->n_phases > GSB_MAX_PHASES ||
        tpl->n_scales < 0 || tpl->n_scales > GSB_MAX_SCALES)
        return set_error(GSB_ERR_INVALID, "template sizes out of range");
    int depth = 0;
    for (int o = 0; o < tpl->n_ops; ++o) {
        const int c = tpl->op_code[o], a = tpl->op_arg[o];
        switch (c) {
          case GSB_OP_LEAF:
            if (a < 0 || a >= tpl->n_leaves) return set_error(GSB_ERR_INVALID, "leaf index out of range");
            ++depth;
            break;
          case GSB_OP_MUL: case GSB_OP_ADD:
            if (depth < 2) return set_error(GSB_ERR_INVALID, "program stack underflow");
            --depth;
            break;
          case GSB_OP_PHASE:
            if (a < 0 || a >= tpl->n_phases || depth < 1)
                return set_error(GSB_ERR_INVALID, "bad PHASE op");
            break;
          case GSB_OP_SCALE:
            if (a < 0 || a >= tpl->n_scales || depth < 1)
                return set_error(GSB_ERR_INVALID, "bad SCALE op");
            break;
          default:
            return set_error(GSB_ERR_INVALID, "unknown opcode");
        }
    }
    if (depth != 1) return set_error(GSB_ERR_INVALID, "program must leave exactly one value");
    for (int l = 0; l < tpl->n_leaves; ++l)
        if (tpl->leaf_type[l] < GSB_GAUSSIAN || tpl->leaf_type[l] > GSB_INTERPOLATED)
            return set_error(GSB_ERR_INVALID, "unknown leaf type");
    return GSB_OK;
}

bool good_fft_size_ok(int n)
{
    if (n < 2) return false;
    while (n % 2 == 0) n /= 2;
    return n == 1 || n == 3;
}

int set_error(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

DeviceState* device_state()
{
    int dev = 0;
    cudaGetDevice(&dev);
    return &g_state[dev & 63];
}

// Record reordering for the FFT-size buckets: gather dst[i] = src[perm[i]] (scatter = 0) or
// scatter dst[perm[i]] = src[i] (scatter = 1), records of `words` 8-byte words, one warp per
// record (consecutive lanes on consecutive words).  Entries of perm outside [0, count) are
// skipped: their destination record is left as it was.
__global__ void permute_records_kernel(unsigned long long* __restrict__ dst,
                                       const unsigned long long* __restrict__ src,
                                       const long long* __restrict__ perm, long long count,
                                       long long words, int scatter)
{
    const long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= count) return;
    const long long p = perm[r];
    if (p < 0 || p >= count) return;
    const unsigned long long* s = src + (scatter ? r : p) * words;
    unsigned long long* d = dst + (scatter ? p : r) * words;
    for (long long w = lane; w < words; w += 32) d[w] = s[w];
}

}  // namespace gsb

using namespace gsb;

extern "C" {

const char* gsb_last_error(void) { return g_err.c_str(); }

int gsb_version(void) { return 1; }

int gsb_init(int device)
{
    std::lock_guard<std::mutex> lock(g_mu);
    GSB_CUDA_CHECK(cudaSetDevice(device));
    DeviceState* st = device_state();
    if (st->ready) return GSB_OK;
    cudaDeviceProp prop;
    GSB_CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return set_error(GSB_ERR_UNSUPPORTED, "libgsb is built for sm_100a (B200); found sm_" +
                                              std::to_string(prop.major * 10 + prop.minor));
    st->sm_count = prop.multiProcessorCount;
    const int rc = ogata_init(st);
    if (rc) return rc;
    st->ready = true;
    return GSB_OK;
}

int gsb_good_fft_size(int input)
{
    // goodFFTSize (src/Image.cpp:1141-1153): the smallest 2^a or 3*2^a (>= 6 for the
    // latter) that is >= input, computed in logs with the same 1e-5 slack.
    if (input <= 2) return 2;
    const double insize = (1. - 1.e-5) * input;
    const double log2n = std::log(2.) * std::ceil(std::log(insize) / std::log(2.));
    double log2n3 = std::log(3.) + std::log(2.) * std::ceil((std::log(insize) - std::log(3.)) / std::log(2.));
    log2n3 = std::max(log2n3, std::log(6.));
    return int(std::ceil(std::exp(std::min(log2n, log2n3)) - 1.e-5));
}

int gsb_tables_create(gsb_tables** out)
{
    if (!out) return set_error(GSB_ERR_INVALID, "null output pointer");
    *out = new gsb_tables();
    return GSB_OK;
}

int gsb_tables_destroy(gsb_tables* t)
{
    if (!t) return GSB_OK;
    cudaFree(t->d_header);
    cudaFree(t->d_node);
    cudaFree(t->d_val);
    cudaFree(t->d_scan);
    cudaFree(t->d_n);
    cudaFree(t->d_status);
    cudaFree(t->d_trunc);
    cudaFree(t->d_dheader);
    cudaFree(t->d_dnode);
    cudaFree(t->d_dval);
    if (t->sersic_exec) cudaGraphExecDestroy(t->sersic_exec);
    if (t->capture_stream) cudaStreamDestroy(t->capture_stream);
    cudaFree(t->d_mheader);
    cudaFree(t->d_mnode);
    cudaFree(t->d_mval);
    cudaFree(t->d_mk);
    cudaFree(t->d_mstatus);
    cudaFree(t->d_images);
    cudaFree(t->d_image_info);
    cudaFree(t->d_k64);
    cudaFree(t->d_k32);
    cudaFree(t->d_krows);
    delete t;
    return GSB_OK;
}

int gsb_sersic_tables_build(gsb_tables* t, const double* h_n, const double* h_trunc_over_r0,
                            int count, const gsb_gsparams* gsp, void* stream)
{
    if (!t || !gsp || (count > 0 && !h_n)) return set_error(GSB_ERR_INVALID, "null argument");
    if (count < 0) return set_error(GSB_ERR_INVALID, "negative count");
    return sersic_tables_build(t, h_n, h_trunc_over_r0, count, gsp, false, (cudaStream_t)stream);
}

int gsb_sersic_tables_build_ex(gsb_tables* t, const double* h_n, const double* h_trunc_over_r0,
                               int count, const gsb_gsparams* gsp, int flags, void* stream)
{
    if (!t || !gsp || (count > 0 && !h_n)) return set_error(GSB_ERR_INVALID, "null argument");
    if (count < 0) return set_error(GSB_ERR_INVALID, "negative count");
    if (flags & ~GSB_TABLES_DN) return set_error(GSB_ERR_INVALID, "unknown table flags");
    return sersic_tables_build(t, h_n, h_trunc_over_r0, count, gsp, (flags & GSB_TABLES_DN) != 0,
                               (cudaStream_t)stream);
}

int gsb_sersic_truncation(int count, const double* h_in, double* h_out, void* stream)
{
    if (count < 0 || (count > 0 && (!h_in || !h_out))) return set_error(GSB_ERR_INVALID, "bad arguments");
    for (int i = 0; i < count; ++i) {
        const double n = h_in[4 * i], size = h_in[4 * i + 1], trunc = h_in[4 * i + 2];
        if (!(n >= 0.3 && n <= 6.2)) return set_error(GSB_ERR_INVALID, "Sersic index out of range [0.3, 6.2]");
        if (!(size > 0.) || !(trunc > 0.)) return set_error(GSB_ERR_INVALID, "size and trunc must be > 0");
        if ((int(h_in[4 * i + 3]) & 3) == 1 && !(trunc > 1.4142135623730951 * size))
            return set_error(GSB_ERR_INVALID, "Sersic truncation must be larger than sqrt(2)*half_light_radius.");
    }
    return sersic_truncation(count, h_in, h_out, (cudaStream_t)stream);
}

int gsb_sersic_tables_info(const gsb_tables* t, double* h_out, int count, void* stream)
{
    if (!t || !h_out) return set_error(GSB_ERR_INVALID, "null argument");
    if (count < 0 || count > t->count) return set_error(GSB_ERR_INVALID, "count exceeds built slots");
    if (count == 0) return GSB_OK;
    GSB_CUDA_CHECK(cudaMemcpyAsync(h_out, t->d_header, sizeof(double) * kSersicHeader * count,
                                   cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return GSB_OK;
}

int gsb_moffat_tables_build(gsb_tables* t, const double* h_beta, const double* h_trunc_over_rd, int count,
                            const gsb_gsparams* gsp, void* stream)
{
    if (!t || !gsp || (count > 0 && (!h_beta || !h_trunc_over_rd))) return set_error(GSB_ERR_INVALID, "null argument");
    if (count < 0) return set_error(GSB_ERR_INVALID, "negative count");
    return moffat_tables_build(t, h_beta, h_trunc_over_rd, count, gsp, (cudaStream_t)stream);
}

int gsb_moffat_tables_info(const gsb_tables* t, double* h_out, int count, void* stream)
{
    if (!t || !h_out) return set_error(GSB_ERR_INVALID, "null argument");
    if (count < 0 || count > t->moffat_count) return set_error(GSB_ERR_INVALID, "count exceeds built slots");
    if (count == 0) return GSB_OK;
    GSB_CUDA_CHECK(cudaMemcpyAsync(h_out, t->d_mheader, sizeof(double) * kMoffatHeader * count,
                                   cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    return GSB_OK;
}

int gsb_moffat_scale_radius(int count, const double* h_in, double* h_out, void* stream)
{
    if (count < 0 || (count > 0 && (!h_in || !h_out))) return set_error(GSB_ERR_INVALID, "bad arguments");
    for (int i = 0; i < count; ++i) {
        const double beta = h_in[3 * i], hlr = h_in[3 * i + 1], trunc = h_in[3 * i + 2];
        if (!(hlr > 0.) || !(trunc >= 0.) || !std::isfinite(beta))
            return set_error(GSB_ERR_INVALID, "half_light_radius must be > 0 and trunc >= 0");
        if (trunc > 0. && !(trunc > 1.4142135623730951 * hlr))
            return set_error(GSB_ERR_INVALID, "Moffat truncation radius must be > sqrt(2) * half_light_radius.");
    }
    return moffat_scale_radius(count, h_in, h_out, (cudaStream_t)stream);
}

int gsb_prepare_leaves(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                       gsb_leaf* d_leaves, const gsb_tables* t, double* d_info, void* stream)
{
    int rc = validate_template(tpl);
    if (rc) return rc;
    if (!gsp || n_stamps < 0 || (n_stamps > 0 && (!d_leaves || !d_info)))
        return set_error(GSB_ERR_INVALID, "null argument");
    return prepare_leaves(tpl, n_stamps, gsp, d_leaves, t, d_info, (cudaStream_t)stream);
}

size_t gsb_draw_workspace_size(int N, int n_stamps, int precision)
{
    if (!good_fft_size_ok(N) || n_stamps <= 0) return 0;
    return draw_workspace_size(N, n_stamps, precision);
}

int gsb_draw_images(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                    const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                    const gsb_stamp* d_stamps, const gsb_tables* t,
                    void* d_out, int out_dtype, int add_to_image, double* d_added_flux,
                    int precision, void* d_workspace, size_t workspace_bytes, void* stream)
{
    int rc = validate_template(tpl);
    if (rc) return rc;
    if (!gsp) return set_error(GSB_ERR_INVALID, "null gsparams");
    if (n_stamps < 0) return set_error(GSB_ERR_INVALID, "negative stamp count");
    if (n_stamps == 0) return GSB_OK;
    if (!d_leaves || !d_stamps || !d_out || (tpl->n_phases && !d_phases) || (tpl->n_scales && !d_scales))
        return set_error(GSB_ERR_INVALID, "null device pointer");
    if (out_dtype != GSB_F32 && out_dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad out_dtype");
    if (precision != GSB_F32 && precision != GSB_F64) return set_error(GSB_ERR_INVALID, "bad precision");
    // The bucket's FFT size is read from the first stamp's geometry by the caller's contract:
    // every stamp in one call has the same N.  It is passed through the stamp array, so read it.
    gsb_stamp first;
    GSB_CUDA_CHECK(cudaMemcpyAsync(&first, d_stamps, sizeof(gsb_stamp), cudaMemcpyDeviceToHost,
                                   (cudaStream_t)stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
    if (!good_fft_size_ok(first.N)) return set_error(GSB_ERR_INVALID, "stamp N is not 2^a or 3*2^a");
    return draw_images(tpl, n_stamps, d_leaves, d_phases, d_scales, d_stamps, t, first.N, d_out,
                       out_dtype, add_to_image, d_added_flux, precision, d_workspace, workspace_bytes,
                       (cudaStream_t)stream);
}

int gsb_draw_bucket(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                    const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                    const gsb_stamp* d_stamps, const gsb_tables* t, int N,
                    void* d_out, int out_dtype, int add_to_image, double* d_added_flux,
                    int precision, void* d_workspace, size_t workspace_bytes, void* stream)
{
    int rc = validate_template(tpl);
    if (rc) return rc;
    if (!gsp) return set_error(GSB_ERR_INVALID, "null gsparams");
    if (n_stamps < 0) return set_error(GSB_ERR_INVALID, "negative stamp count");
    if (n_stamps == 0) return GSB_OK;
    if (!d_leaves || !d_stamps || !d_out || (tpl->n_phases && !d_phases) || (tpl->n_scales && !d_scales))
        return set_error(GSB_ERR_INVALID, "null device pointer");
    if (out_dtype != GSB_F32 && out_dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad out_dtype");
    if (precision != GSB_F32 && precision != GSB_F64) return set_error(GSB_ERR_INVALID, "bad precision");
    if (!good_fft_size_ok(N)) return set_error(GSB_ERR_INVALID, "N is not 2^a or 3*2^a");
    return draw_images(tpl, n_stamps, d_leaves, d_phases, d_scales, d_stamps, t, N, d_out,
                       out_dtype, add_to_image, d_added_flux, precision, d_workspace, workspace_bytes,
                       (cudaStream_t)stream);
}

int gsb_draw_kimages(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                     const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                     const gsb_tables* t, double dk, int kxmin, int kymin, int nkx, int nky,
                     void* d_out, int out_dtype, void* stream)
{
    int rc = validate_template(tpl);
    if (rc) return rc;
    if (!gsp || n_stamps < 0 || nkx < 0 || nky < 0) return set_error(GSB_ERR_INVALID, "bad argument");
    if (n_stamps == 0) return GSB_OK;
    if (!d_leaves || !d_out || (tpl->n_phases && !d_phases) || (tpl->n_scales && !d_scales))
        return set_error(GSB_ERR_INVALID, "null device pointer");
    if (!(dk > 0.)) return set_error(GSB_ERR_INVALID, "dk must be > 0");
    return draw_kimages(tpl, n_stamps, d_leaves, d_phases, d_scales, t, dk, kxmin, kymin, nkx, nky,
                        d_out, out_dtype, (cudaStream_t)stream);
}

int gsb_permute_records(void* d_dst, const void* d_src, const int64_t* d_perm, int64_t count,
                        int64_t record_bytes, int scatter, void* stream)
{
    if (count < 0 || record_bytes <= 0 || record_bytes % 8 || (scatter != 0 && scatter != 1))
        return set_error(GSB_ERR_INVALID, "bad argument");
    if (count == 0) return GSB_OK;
    if (!d_dst || !d_src || !d_perm) return set_error(GSB_ERR_INVALID, "null device pointer");
    if (d_dst == d_src) return set_error(GSB_ERR_INVALID, "d_dst must not alias d_src");
    if ((reinterpret_cast<uintptr_t>(d_dst) | reinterpret_cast<uintptr_t>(d_src) |
         reinterpret_cast<uintptr_t>(d_perm)) & 7)
        return set_error(GSB_ERR_INVALID, "device pointers must be 8-byte aligned");
    const long long threads = 256, warps = threads / 32;
    const long long blocks = (count + warps - 1) / warps;
    permute_records_kernel<<<(unsigned)blocks, (unsigned)threads, 0, (cudaStream_t)stream>>>(
        static_cast<unsigned long long*>(d_dst), static_cast<const unsigned long long*>(d_src),
        reinterpret_cast<const long long*>(d_perm), count, record_bytes / 8, scatter);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GSB_ERR_CUDA, cudaGetErrorString(e));
    return GSB_OK;
}

int gsb_draw_set_variant(int variant) { return draw_set_variant(variant); }

int gsb_exp_fp64(const double* d_x, double* d_y, int n, void* stream)
{
    if (n < 0 || (n > 0 && (!d_x || !d_y))) return set_error(GSB_ERR_INVALID, "bad argument");
    return exp_fp64(d_x, d_y, n, 32, (cudaStream_t)stream);
}

int gsb_exp_fp64_ex(const double* d_x, double* d_y, int n, int table_size, void* stream)
{
    if (n < 0 || (n > 0 && (!d_x || !d_y))) return set_error(GSB_ERR_INVALID, "bad arguments");
    if (table_size != 32 && table_size != 256) return set_error(GSB_ERR_INVALID, "table_size must be 32 or 256");
    if (!device_state()->ready) return set_error(GSB_ERR_INVALID, "gsb_init has not been called");
    return exp_fp64(d_x, d_y, n, table_size, (cudaStream_t)stream);
}

int gsb_draw_tune_report(char* buf, size_t len) { return draw_tune_report(buf, len); }

int gsb_adjoint_grad_count(const gsb_template* tpl)
{
    const int rc = validate_template(tpl);
    if (rc) return rc;
    return adjoint_grad_count(tpl);
}

size_t gsb_adjoint_workspace_size(int N, int n_stamps, int precision)
{
    if (!good_fft_size_ok(N) || n_stamps <= 0) return 0;
    return adjoint_workspace_size(N, n_stamps, precision);
}

int gsb_adjoint_images(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                       const gsb_leaf* d_leaves, const gsb_phase* d_phases, const double* d_scales,
                       const gsb_stamp* d_stamps, const gsb_tables* t, int N,
                       const void* d_cotangent, int cot_dtype, double* d_grad, unsigned int want_mask,
                       int precision, void* d_workspace, size_t workspace_bytes, void* stream)
{
    int rc = validate_template(tpl);
    if (rc) return rc;
    if (!gsp) return set_error(GSB_ERR_INVALID, "null gsparams");
    if (n_stamps < 0) return set_error(GSB_ERR_INVALID, "negative stamp count");
    if (n_stamps == 0) return GSB_OK;
    if (!d_leaves || !d_stamps || !d_cotangent || !d_grad || (tpl->n_phases && !d_phases) ||
        (tpl->n_scales && !d_scales))
        return set_error(GSB_ERR_INVALID, "null device pointer");
    if (cot_dtype != GSB_F32 && cot_dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad cot_dtype");
    if (precision != GSB_F32 && precision != GSB_F64) return set_error(GSB_ERR_INVALID, "bad precision");
    if (!good_fft_size_ok(N)) return set_error(GSB_ERR_INVALID, "N is not 2^a or 3*2^a");
    return adjoint_images(tpl, n_stamps, d_leaves, d_phases, d_scales, d_stamps, t, N, d_cotangent,
                          cot_dtype, d_grad, want_mask, precision, d_workspace, workspace_bytes,
                          (cudaStream_t)stream);
}

}  // extern "C"
