// gsb_draw_images_noalloc: the fused FFT draw for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc or any allocating routine while they
// draw: a host application that hands the GPU a fixed memory budget up front and forbids
// allocation afterwards (for instance a real-time survey pipeline or a plugin living inside
// another program's device-memory pool), or code that must not trigger the implicit
// synchronisation and fragmentation an allocation brings.  gsb_draw_images needs a
// caller-provided scratch slab per CTA when the wrapped k-image does not fit in shared memory
// (N >= 256 in FP32, N >= 192 in FP64); this variant takes that scratch from one fixed array
// compiled into the library instead, and allocates nothing.
//
// Limits and behaviour:
//   * The scratch array is kNoAllocScratchBytes (32 MiB) of device memory, held by every GPU
//     that loads the library until the process exits.
//   * FFT sizes up to 1024 are accepted; larger sizes (the two-kernel large-FFT path) are
//     rejected with GSB_ERR_UNSUPPORTED.  When the slabs of a full grid do not fit, the grid is
//     reduced to the number of slabs that do, so large N runs with fewer CTAs.
//   * The first call on a device looks up the array's device address (cudaGetSymbolAddress)
//     with that device current; make that first call before any stream capture.
//   * Every call shares the one array and nothing in it needs to start at zero (each slab
//     region is fully written before it is read).  Calls whose kernels overlap on the GPU --
//     on different streams, or from different host threads -- race on the array; serialise
//     them on one stream.
#include <mutex>

#include "gsb_draw.cuh"

namespace gsb {

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

// Device-side scratch.  In host code this name is only a handle for cudaGetSymbolAddress,
// never a device address: the address is looked up per device below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocDevice {
    bool ready = false;
    void* ptr = nullptr;
};
NoAllocDevice g_noalloc_dev[64];
std::mutex g_noalloc_mu;

int noalloc_scratch(void** out)
{
    int dev = 0;
    GSB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(GSB_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return set_error(GSB_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                           cudaGetErrorString(e));
        d.ptr = p;
        d.ready = true;
    }
    *out = d.ptr;
    return GSB_OK;
}

template <typename T, int N>
int launch_noalloc(DrawArgs args, cudaStream_t stream)
{
    constexpr bool wsmem = w_fits_smem<T, N>();
    constexpr size_t sm = smem_bytes<T, N>(wsmem);
    int grid = draw_grid<T, N>(args.n_stamps);
    if (!wsmem) {
        constexpr size_t slab = sizeof(Cx<T>) * (size_t)(N / 2 + 1) * (N + 1);
        static_assert(slab <= kNoAllocScratchBytes, "one slab must fit the no-alloc scratch");
        const int fit = int(kNoAllocScratchBytes / slab);
        if (grid > fit) grid = fit;
        void* p = nullptr;
        const int rc = noalloc_scratch(&p);
        if (rc) return rc;
        args.work = p;
    } else {
        args.work = nullptr;
    }
    GSB_CUDA_CHECK(cudaFuncSetAttribute(draw_fused_kernel<T, N, wsmem>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    draw_fused_kernel<T, N, wsmem><<<grid, fused_warps<T, N>() * 32, sm, stream>>>(args);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

template <typename T>
int dispatch_noalloc(int N, const DrawArgs& args, cudaStream_t stream)
{
    switch (N) {
      case 32: return launch_noalloc<T, 32>(args, stream);
      case 48: return launch_noalloc<T, 48>(args, stream);
      case 64: return launch_noalloc<T, 64>(args, stream);
      case 96: return launch_noalloc<T, 96>(args, stream);
      case 128: return launch_noalloc<T, 128>(args, stream);
      case 192: return launch_noalloc<T, 192>(args, stream);
      case 256: return launch_noalloc<T, 256>(args, stream);
      case 384: return launch_noalloc<T, 384>(args, stream);
      case 512: return launch_noalloc<T, 512>(args, stream);
      case 768: return launch_noalloc<T, 768>(args, stream);
      case 1024: return launch_noalloc<T, 1024>(args, stream);
    }
    return set_error(GSB_ERR_UNSUPPORTED, "gsb_draw_images_noalloc supports FFT sizes 2^a or 3*2^a "
                                          "from 32 to 1024; got " + std::to_string(N));
}

int validate_noalloc_template(const gsb_template* tpl)
{
    if (!tpl || tpl->n_ops < 1 || tpl->n_ops > GSB_MAX_OPS || tpl->n_leaves < 1 ||
        tpl->n_leaves > GSB_MAX_LEAVES || tpl->n_phases < 0 || tpl->n_phases > GSB_MAX_PHASES ||
        tpl->n_scales < 0 || tpl->n_scales > GSB_MAX_SCALES)
        return set_error(GSB_ERR_INVALID, "template sizes out of range");
    int depth = 0;
    for (int o = 0; o < tpl->n_ops; ++o) {
        const int c = tpl->op_code[o], a = tpl->op_arg[o];
        if (c == GSB_OP_LEAF) {
            if (a < 0 || a >= tpl->n_leaves) return set_error(GSB_ERR_INVALID, "leaf index out of range");
            ++depth;
        } else if (c == GSB_OP_MUL || c == GSB_OP_ADD) {
            if (depth < 2) return set_error(GSB_ERR_INVALID, "program stack underflow");
            --depth;
        } else if (c == GSB_OP_PHASE) {
            if (a < 0 || a >= tpl->n_phases || depth < 1) return set_error(GSB_ERR_INVALID, "bad PHASE op");
        } else if (c == GSB_OP_SCALE) {
            if (a < 0 || a >= tpl->n_scales || depth < 1) return set_error(GSB_ERR_INVALID, "bad SCALE op");
        } else {
            return set_error(GSB_ERR_INVALID, "unknown opcode");
        }
    }
    if (depth != 1) return set_error(GSB_ERR_INVALID, "program must leave exactly one value");
    for (int l = 0; l < tpl->n_leaves; ++l)
        if (tpl->leaf_type[l] < GSB_GAUSSIAN || tpl->leaf_type[l] > GSB_BOX)
            return set_error(GSB_ERR_INVALID, "unknown leaf type");
    return GSB_OK;
}

}  // namespace

}  // namespace gsb

using namespace gsb;

extern "C" int gsb_draw_images_noalloc(const gsb_template* tpl, int n_stamps, const gsb_gsparams* gsp,
                                       const gsb_leaf* d_leaves, const gsb_phase* d_phases,
                                       const double* d_scales, const gsb_stamp* d_stamps,
                                       const gsb_tables* t, int N, void* d_out, int out_dtype,
                                       int add_to_image, double* d_added_flux, int precision,
                                       void* stream)
{
    int rc = validate_noalloc_template(tpl);
    if (rc) return rc;
    if (!gsp) return set_error(GSB_ERR_INVALID, "null gsparams");
    if (n_stamps < 0) return set_error(GSB_ERR_INVALID, "negative stamp count");
    if (n_stamps == 0) return GSB_OK;
    if (!d_leaves || !d_stamps || !d_out || (tpl->n_phases && !d_phases) || (tpl->n_scales && !d_scales))
        return set_error(GSB_ERR_INVALID, "null device pointer");
    if (out_dtype != GSB_F32 && out_dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "bad out_dtype");
    if (precision != GSB_F32 && precision != GSB_F64) return set_error(GSB_ERR_INVALID, "bad precision");
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
    args.add = add_to_image;
    args.added_flux = d_added_flux;
    args.work = nullptr;
    return precision == GSB_F64 ? dispatch_noalloc<double>(N, args, (cudaStream_t)stream)
                                : dispatch_noalloc<float>(N, args, (cudaStream_t)stream);
}
