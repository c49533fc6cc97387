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
//   * Every stamp's FFT size must equal the N argument.  A small check kernel compares them
//     first and records a mismatch in a status word that is also static device memory; the
//     call reads that word back (so it returns once the stream has reached the check) and
//     refuses the draw with GSB_ERR_INVALID.
//   * Programs with InterpolatedImage leaves are accepted as in gsb_draw_images; programs
//     without them run the kernel instance compiled without the image-leaf code, as there.
//   * The first call on a device looks up the device addresses of the array and of the
//     status word (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.  The addresses are kept for the life of the process, so the
//     library must not be used on a device after cudaDeviceReset.
//   * Every call shares the one array and nothing in it needs to start at zero (each slab
//     region is fully written before it is read; the status word is cleared by each call).
//     Calls whose kernels overlap on the GPU -- on different streams, or from different host
//     threads -- race on the array; serialise them on one stream.
#include <mutex>

#include "gsb_draw.cuh"

namespace gsb {

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

// Device-side scratch.  In host code this name is only a handle for cudaGetSymbolAddress,
// never a device address: the address is looked up per device below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
// Stamp-geometry check result of the current call (nonzero: a stamp's N differs from N).
static __device__ int g_noalloc_status;

struct NoAllocDevice {
    bool ready = false;
    void* ptr = nullptr;
    int* status = nullptr;
};
NoAllocDevice g_noalloc_dev[64];
std::mutex g_noalloc_mu;

int noalloc_scratch(void** out, int** status)
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
        void* q = nullptr;
        const cudaError_t e2 = cudaGetSymbolAddress(&q, g_noalloc_status);
        if (e2 != cudaSuccess)
            return set_error(GSB_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc status): ") +
                                           cudaGetErrorString(e2));
        d.ptr = p;
        d.status = static_cast<int*>(q);
        d.ready = true;
    }
    *out = d.ptr;
    if (status) *status = d.status;
    return GSB_OK;
}

__global__ void noalloc_check_kernel(const gsb_stamp* stamps, int n_stamps, int N, int* status)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n_stamps && stamps[s].N != N) atomicOr(status, 1);
}

// Every stamp's N against the call's N, on the device; the answer is read back before drawing.
int noalloc_check_stamps(const gsb_stamp* d_stamps, int n_stamps, int N, int* d_status, cudaStream_t stream)
{
    GSB_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), stream));
    noalloc_check_kernel<<<(n_stamps + 255) / 256, 256, 0, stream>>>(d_stamps, n_stamps, N, d_status);
    GSB_CUDA_CHECK(cudaGetLastError());
    int h = 0;
    GSB_CUDA_CHECK(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    if (h) return set_error(GSB_ERR_INVALID, "gsb_draw_images_noalloc: a stamp's FFT size differs from N = " +
                                             std::to_string(N));
    return GSB_OK;
}

template <typename T, int N, bool II>
int launch_noalloc_ii(const DrawArgs& args, int grid, cudaStream_t stream)
{
    constexpr bool wsmem = w_fits_smem<T, N>();
    constexpr size_t sm = smem_bytes<T, N>(wsmem);
    GSB_CUDA_CHECK(cudaFuncSetAttribute(draw_fused_kernel<T, N, wsmem, II>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    draw_fused_kernel<T, N, wsmem, II><<<grid, fused_warps<T, N>() * 32, sm, stream>>>(args);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

template <typename T, int N>
int launch_noalloc(DrawArgs args, cudaStream_t stream)
{
    constexpr bool wsmem = w_fits_smem<T, N>();
    int grid = draw_grid<T, N>(args.n_stamps);
    void* p = nullptr;
    int* status = nullptr;
    int rc = noalloc_scratch(&p, &status);
    if (rc) return rc;
    rc = noalloc_check_stamps(args.stamps, args.n_stamps, N, status, stream);
    if (rc) return rc;
    if (!wsmem) {
        constexpr size_t slab = sizeof(Cx<T>) * (size_t)(N / 2 + 1) * (N + 1);
        static_assert(slab <= kNoAllocScratchBytes, "one slab must fit the no-alloc scratch");
        const int fit = int(kNoAllocScratchBytes / slab);
        if (grid > fit) grid = fit;
        args.work = p;
    } else {
        args.work = nullptr;
    }
    // programs without image leaves run the instance compiled without their code
    return has_image_leaves(args.tpl) ? launch_noalloc_ii<T, N, true>(args, grid, stream)
                                      : launch_noalloc_ii<T, N, false>(args, grid, stream);
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
    int rc = validate_template(tpl);
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
