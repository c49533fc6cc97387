// Public draw entry points: dispatch to the per-size kernel instantiations.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

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

// ---- draw-variant autotuner ------------------------------------------------------------
// For a bucket of FFT size N <= 1024 two kernels are available: the fused kernel (one CTA per
// stamp, persistent) and the split pair of the large-FFT path (column CTAs, then row CTAs, the
// wrapped k-image through HBM).  The fused kernel wins when the bucket fills the GPU; for a
// bucket of a few large stamps the split pair spreads each stamp over hundreds of CTAs.  The
// first draw of a (device, precision, N, log2 stamp count) class times both on the real inputs
// (when the call overwrites its output and the stream is not capturing) and keeps the faster;
// otherwise a size rule decides.
namespace {

constexpr size_t kSplitWorkBudget = size_t(256) << 20;   // scratch cap of a split candidate

struct TuneKey {
    int dev, prec, N, cls;
    bool operator<(const TuneKey& o) const
    {
        return dev != o.dev ? dev < o.dev : prec != o.prec ? prec < o.prec : N != o.N ? N < o.N : cls < o.cls;
    }
};

struct TuneEntry { int variant; float ms_fused, ms_split; bool timed; };

std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;
int g_force_variant = 0;   // 0 automatic, 1 fused, 2 split

int ilog2(int n) { int c = 0; while (n > 1) { n >>= 1; ++c; } return c; }

bool split_candidate(int N, int n_stamps)
{
    DeviceState* st = device_state();
    return N >= 192 && N <= 1024 && n_stamps < 2 * st->sm_count;
}

size_t split_workspace(int N, int n_stamps, int precision)
{
    const size_t slab = (precision == GSB_F64 ? 16 : 8) * (size_t)(N / 2 + 1) * N;
    const size_t k = std::max<size_t>(1, std::min<size_t>((size_t)n_stamps, kSplitWorkBudget / slab));
    return k * slab;
}

int rule_variant(int N, int n_stamps)
{
    DeviceState* st = device_state();
    return (N >= 256 && 4 * n_stamps < st->sm_count) ? 1 : 0;
}

}  // namespace

int draw_set_variant(int v)
{
    if (v < 0 || v > 2) return set_error(GSB_ERR_INVALID, "variant must be 0 (automatic), 1 (fused) or 2 (split)");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_force_variant = v;
    return GSB_OK;
}

int draw_tune_report(char* buf, size_t len)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::string out;
    for (const auto& kv : g_tune) {
        char line[160];
        snprintf(line, sizeof(line), "dev=%d prec=%s N=%d stamps=2^%d variant=%s fused_ms=%.4f split_ms=%.4f%s\n",
                 kv.first.dev, kv.first.prec == GSB_F64 ? "f64" : "f32", kv.first.N, kv.first.cls,
                 kv.second.variant ? "split" : "fused", kv.second.ms_fused, kv.second.ms_split,
                 kv.second.timed ? "" : " (size rule)");
        out += line;
    }
    if (buf && len) {
        const size_t n = std::min(len - 1, out.size());
        memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return int(out.size());
}

size_t draw_workspace_size(int N, int n_stamps, int precision)
{
    if (is_large_fft(N)) return large_workspace_size(N, n_stamps, precision);
    size_t b = 0;
    if (precision == GSB_F64) {
        if (!(fused_workspace_f64_small(N, n_stamps, &b) || fused_workspace_f64_large(N, n_stamps, &b))) return 0;
    } else {
        if (!(fused_workspace_f32_small(N, n_stamps, &b) || fused_workspace_f32_large(N, n_stamps, &b))) return 0;
    }
    if (split_candidate(N, n_stamps)) b = std::max(b, split_workspace(N, n_stamps, precision));
    return b;
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
    auto fused = [&]() -> int {
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
    };
    auto split = [&]() -> int { return draw_large(args, N, precision, d_work, work_bytes, stream); };
    const bool cand = split_candidate(N, n_stamps) && d_work && work_bytes >= split_workspace(N, n_stamps, precision);
    int force;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        force = g_force_variant;
    }
    if (force == 1 || (force == 0 && !cand)) return fused();
    if (force == 2) {
        if (N < 192 || !d_work || work_bytes < split_workspace(N, n_stamps, precision))
            return fused();
        return split();
    }
    int dev = 0;
    cudaGetDevice(&dev);
    const TuneKey key{dev, precision, N, ilog2(n_stamps)};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) return it->second.variant ? split() : fused();
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    GSB_CUDA_CHECK(cudaStreamIsCapturing(stream, &cap));
    if (add || cap != cudaStreamCaptureStatusNone) {
        // cannot time here (the output accumulates, or the stream is being captured: then the
        // fused kernel, whose set-up needs no allocation)
        const int v = cap != cudaStreamCaptureStatusNone ? 0 : rule_variant(N, n_stamps);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = TuneEntry{v, 0.f, 0.f, false};
        return v ? split() : fused();
    }
    // time both on this call's inputs, after one untimed run of each (the first launch of a
    // kernel also loads it); each run writes the complete output, the last one stands
    int rc = fused();
    if (!rc) rc = split();
    if (rc) return rc;
    cudaEvent_t e0, e1, e2;
    GSB_CUDA_CHECK(cudaEventCreate(&e0));
    GSB_CUDA_CHECK(cudaEventCreate(&e1));
    GSB_CUDA_CHECK(cudaEventCreate(&e2));
    if (cudaEventRecord(e0, stream) != cudaSuccess) rc = set_error(GSB_ERR_CUDA, "cudaEventRecord");
    if (!rc) rc = fused();
    if (!rc && cudaEventRecord(e1, stream) != cudaSuccess) rc = set_error(GSB_ERR_CUDA, "cudaEventRecord");
    if (!rc) rc = split();
    if (!rc && cudaEventRecord(e2, stream) != cudaSuccess) rc = set_error(GSB_ERR_CUDA, "cudaEventRecord");
    float ms_f = 0.f, ms_s = 0.f;
    if (!rc && cudaEventSynchronize(e2) == cudaSuccess) {
        cudaEventElapsedTime(&ms_f, e0, e1);
        cudaEventElapsedTime(&ms_s, e1, e2);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = TuneEntry{ms_s < ms_f ? 1 : 0, ms_f, ms_s, true};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
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
