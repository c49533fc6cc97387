// Large-FFT drawing path (1024 < N <= 16384): two kernels per chunk of stamps.
//
//   large_col_kernel: one CTA per (column group, stamp).  For each column kx = 0..N/2 it
//     builds the wrapped k-values of all N rows (alias sums of the program, as in the fused
//     kernel), inverse-transforms them with a block-wide Stockham FFT in shared memory and
//     stores the column into the stamp's slab W (column-major, coalesced).
//   large_row_kernel: one CTA per (row pair, stamp).  It gathers two image rows of W,
//     packs them as one complex row (row1 + i row2, Hermitian-extended in kx), transforms it,
//     writes the pixels inside the stamp scaled by 1/N^2 and adds the compensated flux sum.
// The slab W is the only HBM round trip; the chunk size keeps it inside the workspace.
#include <algorithm>
#include <map>
#include <mutex>

#include "gsb_draw.cuh"

namespace gsb {

static __global__ void twiddle_kernel(double2* tw, int N)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    double s, c;
    sincospi(2.0 * m / N, &s, &c);
    tw[m] = make_double2(c, s);
}

static std::map<int, double2*>& twiddle_cache()
{
    static std::map<int, double2*> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    return cache[dev & 63];
}

// exp(+2 pi i m / N), m < N, in FP64: built once per (device, N) and kept for the process.
int fft_twiddles(int N, cudaStream_t stream, const double2** out)
{
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    auto& c = twiddle_cache();
    auto it = c.find(N);
    if (it != c.end()) { *out = it->second; return GSB_OK; }
    double2* tw = nullptr;
    GSB_CUDA_CHECK(cudaMalloc(&tw, sizeof(double2) * N));
    twiddle_kernel<<<(N + 255) / 256, 256, 0, stream>>>(tw, N);
    GSB_CUDA_CHECK(cudaGetLastError());
    GSB_CUDA_CHECK(cudaStreamSynchronize(stream));
    c[N] = tw;
    *out = tw;
    return GSB_OK;
}

namespace {

constexpr int kLargeThreads = 1024;

struct LargeArgs {
    DrawArgs a;          // leaves/phases/scales/stamps already offset to the chunk
    int N;
    const double2* tw;
    void* W;             // n_stamps slabs of (N/2+1) x N complex
    int cache_bytes;     // shared memory for the per-stamp caches (factored program)
};

template <typename T, int THREADS, bool II>
__global__ void __launch_bounds__(THREADS) large_col_kernel(const __grid_constant__ LargeArgs la)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StampSmem& S = *reinterpret_cast<StampSmem*>(smem_raw);
    Cx<T>* buf = reinterpret_cast<Cx<T>*>(smem_raw + ((sizeof(StampSmem) + 15) & ~size_t(15)));
    const DrawArgs& a = la.a;
    const int N = la.N, H = N / 2 + 1;
    unsigned char* cache = reinterpret_cast<unsigned char*>(buf + N);
    const int s = blockIdx.y;
    const double dk = 2. * kPi / N;
    load_stamp(S, a.tpl, s, a.leaves, a.phases, a.scales, a.stamps, a.sersic_header, a.sersic_node,
               a.sersic_stride, 1. / N);
    __syncthreads();
    const int Nk = S.geom.Nk, hk = Nk / 2;
    const GridRef g{dk, 0, -hk, hk + 1, Nk + 1};
    if (threadIdx.x == 0) plan_caches<T, II>(S, a.tpl, Nk, 0u, la.cache_bytes);
    __syncthreads();
    fill_caches<T, II>(S, a.tpl, cache, dk, Nk);
    __syncthreads();
    const bool factored = S.xy_cache >= 0, fast = S.regstack;
    Cx<T>* W = reinterpret_cast<Cx<T>*>(la.W) + (size_t)s * H * N;
    for (int c = blockIdx.x; c < H; c += gridDim.x) {
        const int alo = ceil_div(-hk - c, N), ahi = floor_div(hk - c, N);
        for (int r = threadIdx.x; r < N; r += blockDim.x) {
            const int kyc = r < N / 2 ? r : r - N;
            const int blo = ceil_div(-hk - kyc, N), bhi = floor_div(hk - kyc, N);
            Cx<T> acc = cx<T>(T(0), T(0)), comp = acc;     // Kahan-compensated fold
            for (int ia = alo; ia <= ahi; ++ia) {
                const int kx = c + ia * N;
                for (int ib = blo; ib <= bhi; ++ib) {
                    const int ky = kyc + ib * N;
                    const bool pos = kx >= 0;
                    const int ii = pos ? kx : -kx, jj = pos ? ky : -ky;
                    const Cx<T> v = factored ? eval_factored<T, II>(a.tpl, S, cache, dk, ii, jj, g)
                                    : fast ? eval_fast<T, II>(a.tpl, S, cache, dk, ii, jj, g)
                                           : eval_program<T, II>(a.tpl, S, dk, ii, jj, g);
                    kahan_add<T>(acc, comp, pos ? v : cconj<T>(v));
                }
            }
            buf[r] = acc;
        }
        __syncthreads();
        block_fft<T, +1>(buf, N, la.tw);
        for (int r = threadIdx.x; r < N; r += blockDim.x) W[(size_t)c * N + r] = buf[r];
        __syncthreads();
    }
}

template <typename T, int THREADS>
__global__ void __launch_bounds__(THREADS) large_row_kernel(const __grid_constant__ LargeArgs la)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    StampSmem& S = *reinterpret_cast<StampSmem*>(smem_raw);
    Cx<T>* buf = reinterpret_cast<Cx<T>*>(smem_raw + ((sizeof(StampSmem) + 15) & ~size_t(15)));
    const DrawArgs& a = la.a;
    const int N = la.N, H = N / 2 + 1;
    const int s = blockIdx.y;
    if (threadIdx.x == 0) S.geom = a.stamps[s];
    __syncthreads();
    const gsb_stamp G = S.geom;
    const Cx<T>* W = reinterpret_cast<const Cx<T>*>(la.W) + (size_t)s * H * N;
    const T inv_n2 = T(1) / (T(N) * T(N));
    const int npairs = (G.ny + 1) / 2;
    double fsum = 0., fcomp = 0.;
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        const int py1 = G.ymin + 2 * p;
        const bool two = 2 * p + 1 < G.ny;
        const int y1 = pmod(py1, N), y2 = pmod(py1 + 1, N);
        for (int kx = threadIdx.x; kx < N; kx += blockDim.x) {
            Cx<T> a1, a2;
            if (kx < H) {
                a1 = W[(size_t)kx * N + y1];
                a2 = two ? W[(size_t)kx * N + y2] : cx<T>(T(0), T(0));
            } else {
                a1 = cconj<T>(W[(size_t)(N - kx) * N + y1]);
                a2 = two ? cconj<T>(W[(size_t)(N - kx) * N + y2]) : cx<T>(T(0), T(0));
            }
            buf[kx] = cx<T>(a1.x - a2.y, a1.y + a2.x);
        }
        __syncthreads();
        block_fft<T, +1>(buf, N, la.tw);
        const long long row1 = G.out_offset + (long long)(2 * p) * G.nx;
        for (int i = threadIdx.x; i < G.nx; i += blockDim.x) {
            const Cx<T> v = buf[pmod(G.xmin + i, N)];
            const T v1 = v.x * inv_n2;
            store_pixel<T>(a.out, a.out_dtype, a.add, row1 + i, v1);
            double x = double(v1), t = fsum + x;
            fcomp += fabs(fsum) >= fabs(x) ? (fsum - t) + x : (x - t) + fsum;
            fsum = t;
            if (two) {
                const T v2 = v.y * inv_n2;
                store_pixel<T>(a.out, a.out_dtype, a.add, row1 + G.nx + i, v2);
                x = double(v2);
                t = fsum + x;
                fcomp += fabs(fsum) >= fabs(x) ? (fsum - t) + x : (x - t) + fsum;
                fsum = t;
            }
        }
        __syncthreads();
    }
    if (a.added_flux) {
        double v = fsum + fcomp;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        __shared__ double part[kLargeThreads / 32];
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += part[w];
            atomicAdd(&a.added_flux[s], tot);
        }
    }
}

template <typename T>
size_t slab_bytes(int N) { return sizeof(Cx<T>) * (size_t)(N / 2 + 1) * N; }

template <typename T>
size_t large_smem() { return ((sizeof(StampSmem) + 15) & ~size_t(15)); }

template <typename T, int THREADS>
int launch_large_t(const DrawArgs& args, int N, void* work, size_t work_bytes, cudaStream_t stream)
{
    const size_t slab = slab_bytes<T>(N);
    if (!work || work_bytes < slab) return set_error(GSB_ERR_INVALID, "draw workspace too small");
    const size_t base = large_smem<T>() + sizeof(Cx<T>) * N;
    if (base > kSmemLimit) return set_error(GSB_ERR_UNSUPPORTED, "FFT size too large for this precision");
    // the rest of shared memory (up to 192 KB) holds the per-stamp caches of the column kernel
    const size_t room = kSmemLimit - base > 1024 ? kSmemLimit - base - 1024 : 0;
    const int cache_bytes = int(std::min<size_t>(room, 192 * 1024) & ~size_t(15));
    const size_t sm = base + cache_bytes;
    const double2* tw = nullptr;
    int rc = fft_twiddles(N, stream, &tw);
    if (rc) return rc;
    // programs without image leaves run the column kernel compiled without their code
    const bool ii = has_image_leaves(args.tpl);
    if (ii)
        GSB_CUDA_CHECK(cudaFuncSetAttribute(large_col_kernel<T, THREADS, true>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    else
        GSB_CUDA_CHECK(cudaFuncSetAttribute(large_col_kernel<T, THREADS, false>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    GSB_CUDA_CHECK(cudaFuncSetAttribute(large_row_kernel<T, THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(base)));
    const int chunk = int(std::max<size_t>(1, std::min<size_t>(work_bytes / slab, 65535)));
    DeviceState* st = device_state();
    if (args.added_flux)
        GSB_CUDA_CHECK(cudaMemsetAsync(args.added_flux, 0, sizeof(double) * args.n_stamps, stream));
    for (int s0 = 0; s0 < args.n_stamps; s0 += chunk) {
        const int n = std::min(chunk, args.n_stamps - s0);
        LargeArgs la;
        la.a = args;
        la.a.n_stamps = n;
        la.a.leaves = args.leaves + (size_t)s0 * args.tpl.n_leaves;
        la.a.phases = args.phases ? args.phases + (size_t)s0 * args.tpl.n_phases : nullptr;
        la.a.scales = args.scales ? args.scales + (size_t)s0 * args.tpl.n_scales : nullptr;
        la.a.stamps = args.stamps + s0;
        la.a.added_flux = args.added_flux ? args.added_flux + s0 : nullptr;
        la.N = N;
        la.tw = tw;
        la.W = work;
        la.cache_bytes = cache_bytes;
        const int cols = N / 2 + 1;
        const int gx = std::max(1, std::min(cols, (2 * st->sm_count + n - 1) / n));
        if (ii) large_col_kernel<T, THREADS, true><<<dim3(gx, n), THREADS, sm, stream>>>(la);
        else large_col_kernel<T, THREADS, false><<<dim3(gx, n), THREADS, sm, stream>>>(la);
        GSB_CUDA_CHECK(cudaGetLastError());
        const int gr = std::max(1, std::min(N / 2, (2 * st->sm_count + n - 1) / n));
        large_row_kernel<T, THREADS><<<dim3(gr, n), THREADS, base, stream>>>(la);
        GSB_CUDA_CHECK(cudaGetLastError());
    }
    return GSB_OK;
}

// Threads per CTA: one per row, 256 to 1024.
template <typename T>
int launch_large(const DrawArgs& args, int N, void* work, size_t work_bytes, cudaStream_t stream)
{
    if (N <= 256) return launch_large_t<T, 256>(args, N, work, work_bytes, stream);
    if (N <= 512) return launch_large_t<T, 512>(args, N, work, work_bytes, stream);
    return launch_large_t<T, kLargeThreads>(args, N, work, work_bytes, stream);
}

}  // namespace

bool is_large_fft(int N) { return N > 1024 && N <= 16384; }

size_t large_workspace_size(int N, int n_stamps, int precision)
{
    const size_t slab = precision == GSB_F64 ? slab_bytes<double>(N) : slab_bytes<float>(N);
    // up to 8 GiB of slabs per chunk, at least one stamp
    const size_t budget = size_t(8) << 30;
    const size_t k = std::max<size_t>(1, std::min<size_t>((size_t)n_stamps, budget / slab));
    return k * slab;
}

int draw_large(const DrawArgs& args, int N, int precision, void* work, size_t work_bytes,
               cudaStream_t stream)
{
    return precision == GSB_F64 ? launch_large<double>(args, N, work, work_bytes, stream)
                                : launch_large<float>(args, N, work, work_bytes, stream);
}

}  // namespace gsb
