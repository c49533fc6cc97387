// Adjoint of the split large-FFT draw (N = 1536 .. 16384, gsb_draw_large.cu), by stamps.
//
// The same reverse mode as adjoint_fused_kernel (gsb_adjoint.cuh), with the transforms of the
// large path: for a loss L with image cotangent G,
//     dL = sum_{c,r} (w_c / N^2) Re(Ghat(c, r) dX(c, r)),  Ghat = forward-sign DFT of G placed
//     at the pixels' (x mod N, y mod N),
// where X is the wrapped k-image.  Three kernels per chunk of stamps:
//   adj_large_row_kernel  pairs of cotangent rows, one block-wide FFT per pair, unpacked into
//                         the half-plane columns c = 0..N/2 of a per-stamp slab W[c][y];
//   adj_large_col_kernel  per column c (blocks stride over columns): the FFT along y gives
//                         Ghat(c, .), then every alias of every cell runs the program in reverse
//                         (adjoint_point_factored / adjoint_range), each thread accumulating its
//                         terms; one reduction per block into the FP64 gradients;
//   adj_large_finalize_kernel  the hlr chain rule of Sersic leaves and the want mask.
#include "gsb_adjoint.cuh"

namespace gsb {

int fft_twiddles(int N, cudaStream_t stream, const double2** out);
bool is_large_fft(int N);

namespace {

struct AdjLargeArgs {
    AdjArgs a;           // leaves / phases / scales / stamps / grad offset to the chunk
    int N;
    const double2* tw;   // exp(+2 pi i m / N), FP64
    void* W;             // per-stamp slabs of (N/2 + 1) x N complex
    int cache_bytes;     // shared memory for the per-stamp caches of the column kernel
};

template <typename T, int THREADS>
__global__ void __launch_bounds__(THREADS) adj_large_row_kernel(const __grid_constant__ AdjLargeArgs la)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cx<T>* buf = reinterpret_cast<Cx<T>*>(smem_raw);
    __shared__ gsb_stamp G;
    const AdjArgs& a = la.a;
    const int N = la.N, H = N / 2 + 1;
    const int s = blockIdx.y;
    if (threadIdx.x == 0) G = a.stamps[s];
    __syncthreads();
    Cx<T>* W = reinterpret_cast<Cx<T>*>(la.W) + (size_t)s * H * N;
    const int npairs = (G.ny + 1) / 2;
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        const bool two = 2 * p + 1 < G.ny;
        for (int x = threadIdx.x; x < N; x += blockDim.x) buf[x] = cx<T>(T(0), T(0));
        __syncthreads();
        const long long row1 = G.out_offset + (long long)(2 * p) * G.nx;
        for (int i = threadIdx.x; i < G.nx; i += blockDim.x) {
            const T g1 = load_cot<T>(a.cot, a.cot_dtype, row1 + i);
            const T g2 = two ? load_cot<T>(a.cot, a.cot_dtype, row1 + G.nx + i) : T(0);
            buf[pmod(G.xmin + i, N)] = cx<T>(g1, g2);
        }
        __syncthreads();
        block_fft<T, +1>(buf, N, la.tw);
        const int y1 = pmod(G.ymin + 2 * p, N), y2 = pmod(G.ymin + 2 * p + 1, N);
        for (int c = threadIdx.x; c < H; c += blockDim.x) {
            const Cx<T> z = buf[c];
            const Cx<T> zm = buf[c == 0 ? 0 : N - c];
            W[(size_t)c * N + y1] = cx<T>(T(0.5) * (z.x + zm.x), T(0.5) * (z.y - zm.y));
            if (two) W[(size_t)c * N + y2] = cx<T>(T(0.5) * (z.y + zm.y), T(0.5) * (zm.x - z.x));
        }
        __syncthreads();
    }
}

template <typename T, int THREADS, bool II>
__global__ void __launch_bounds__(THREADS) adj_large_col_kernel(const __grid_constant__ AdjLargeArgs la)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const AdjArgs& a = la.a;
    const int N = la.N, H = N / 2 + 1;
    AdjSmem& A = *reinterpret_cast<AdjSmem*>(smem_raw);
    StampSmem& S = A.S;
    size_t off = (sizeof(AdjSmem) + 15) & ~size_t(15);
    Cx<T>* buf = reinterpret_cast<Cx<T>*>(smem_raw + off);
    off += sizeof(Cx<T>) * N;
    unsigned char* cache = smem_raw + ((off + 15) & ~size_t(15));
    const int s = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const double dk = 2. * kPi / N;
    const T inv_n2 = T(1) / (T(N) * T(N));
    const int ng = grad_count(a.tpl);
    if (threadIdx.x == 0) program_children(a.tpl, A.child1, A.child2);
    load_stamp(S, a.tpl, s, a.leaves, a.phases, a.scales, a.stamps, a.sersic_header, a.sersic_node,
               a.sersic_stride, 1. / N);
    if (threadIdx.x < a.tpl.n_leaves && a.sersic_dheader &&
        a.tpl.leaf_type[threadIdx.x] == GSB_SERSIC) {
        const int t = a.leaves[(size_t)s * a.tpl.n_leaves + threadIdx.x].table;
        const double* D = a.sersic_dheader + (size_t)t * kSersicDHeader;
        SersicDnView& v = A.dn[threadIdx.x];
        v.dkd2 = D[kSD_DKD2];
        v.dkd4 = D[kSD_DKD4];
        v.dhigha = D[kSD_DHIGHA];
        v.dhighb = D[kSD_DHIGHB];
        v.dlnre = D[kSD_DLNRE];
        v.dfront = D[kSD_DFRONT];
        v.node = a.sersic_dnode + (size_t)t * a.sersic_stride;
    }
    for (int k = threadIdx.x; k < ng; k += blockDim.x) A.gacc[k] = 0.;
    __syncthreads();
    const gsb_stamp& G = S.geom;
    const int Nk = G.Nk, hk = Nk / 2;
    const GridRef g{dk, 0, -hk, hk + 1, Nk + 1};
    if (threadIdx.x == 0) plan_caches<T, II>(S, a.tpl, Nk, a.want, la.cache_bytes);
    __syncthreads();
    fill_caches<T, II>(S, a.tpl, cache, dk, Nk);
    __syncthreads();
    const bool factored = S.xy_cache >= 0 && S.n_atoms <= kAdjAtoms;
    bool subtree = !factored;
    if (factored)
        for (int t = 0; t < S.n_atoms; ++t)
            subtree |= (S.atom_kind[t] == kAtomRange || S.atom_kind[t] == kAtomSum) &&
                       S.atom_o1[t] - S.atom_o0[t] > 1;
    const Cx<T>* W = reinterpret_cast<const Cx<T>*>(la.W) + (size_t)s * H * N;
    T acc[kMaxGrad];
    T ga[kAdjAtoms][kGradPerPhase];
    if (subtree)
        for (int k = 0; k < ng; ++k) acc[k] = T(0);
#pragma unroll
    for (int t = 0; t < kAdjAtoms; ++t)
#pragma unroll
        for (int e = 0; e < kGradPerPhase; ++e) ga[t][e] = T(0);
    for (int c = blockIdx.x; c < H; c += gridDim.x) {
        for (int y = threadIdx.x; y < N; y += blockDim.x)
            buf[y] = pmod(y - G.ymin, N) < G.ny ? W[(size_t)c * N + y] : cx<T>(T(0), T(0));
        __syncthreads();
        block_fft<T, +1>(buf, N, la.tw);
        const T wc = (c == 0 || 2 * c == N) ? inv_n2 : T(2) * inv_n2;
        const int alo = ceil_div(-hk - c, N), ahi = floor_div(hk - c, N);
        for (int r = threadIdx.x; r < N; r += blockDim.x) {
            const Cx<T> gh = cscale<T>(buf[r], wc);
            const int kyc = r < N / 2 ? r : r - N;
            const int blo = ceil_div(-hk - kyc, N), bhi = floor_div(hk - kyc, N);
            for (int ia = alo; ia <= ahi; ++ia) {
                const int kx = c + ia * N;
                for (int ib = blo; ib <= bhi; ++ib) {
                    const int ky = kyc + ib * N;
                    const bool pos = kx >= 0;
                    // an alias taken as conj(F(-k)) contributes Re(Ghat conj(dF)) = Re(conj(Ghat) dF)
                    if (factored)
                        adjoint_point_factored<T, II>(a.tpl, A, cache, a.want, dk, pos ? kx : -kx,
                                                      pos ? ky : -ky, g, pos ? gh : cconj<T>(gh), ga, acc);
                    else
                        adjoint_range<T, II>(a.tpl, A, dk, pos ? kx : -kx, pos ? ky : -ky, g,
                                             pos ? gh : cconj<T>(gh), acc, 0, a.tpl.n_ops);
                }
            }
        }
        __syncthreads();
    }
    // one reduction per block: warp shuffles in FP64, shared atomics, then the global sums
    if (subtree) {
        for (int k = 0; k < ng; ++k) {
            double v = double(acc[k]);
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) atomicAdd(&A.gacc[k], v);
        }
    }
    if (factored) {
        const int pbase = kGradPerLeaf * a.tpl.n_leaves;
        const int sbase = pbase + kGradPerPhase * a.tpl.n_phases;
#pragma unroll
        for (int t = 0; t < kAdjAtoms; ++t) {
            if (t >= S.n_atoms) break;
            const int kind = S.atom_kind[t];
            int base, cnt;
            if (kind == kAtomPhase) { base = pbase + kGradPerPhase * S.atom_arg[t]; cnt = kGradPerPhase; }
            else if (kind == kAtomScale) { base = sbase + S.atom_arg[t]; cnt = 1; }
            else if (S.atom_o1[t] - S.atom_o0[t] == 1 && want_leaf(a.want, S.atom_arg[t])) {
                base = kGradPerLeaf * S.atom_arg[t]; cnt = kGradPerLeaf;
            } else continue;
#pragma unroll
            for (int e = 0; e < kGradPerPhase; ++e) {
                if (e >= cnt) break;
                double v = double(ga[t][e]);
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) atomicAdd(&A.gacc[base + e], v);
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < ng; k += blockDim.x)
        if (A.gacc[k] != 0.) atomicAdd(&a.grad[(size_t)s * ng + k], A.gacc[k]);
}

// Sersic leaves given by half-light radius: r0 = hlr / r_e(n), so at fixed hlr d/dn picks up
// -d ln r_e/dn * d/d ln r0, and d/d ln r0 = sum_ij J_ij d/dJ_ij; then entries of records
// outside the want mask are zeroed.  One block per stamp.
__global__ void adj_large_finalize_kernel(const __grid_constant__ AdjArgs a)
{
    const int s = blockIdx.x;
    const int ng = grad_count(a.tpl);
    double* gr = a.grad + (size_t)s * ng;
    const int l = threadIdx.x;
    if (l < a.tpl.n_leaves && want_leaf(a.want, l) && a.tpl.leaf_type[l] == GSB_SERSIC && a.sersic_dheader) {
        const gsb_leaf& L = a.leaves[(size_t)s * a.tpl.n_leaves + l];
        if (L.flags & GSB_LEAF_SIZE_IS_HLR) {
            double* gl = gr + kGradPerLeaf * l;
            const double glnr0 = L.jac[0] * gl[1] + L.jac[1] * gl[2] + L.jac[2] * gl[3] + L.jac[3] * gl[4];
            gl[5] -= a.sersic_dheader[(size_t)L.table * kSersicDHeader + kSD_DLNRE] * glnr0;
        }
    }
    __syncthreads();
    const int pbase = kGradPerLeaf * a.tpl.n_leaves;
    const int sbase = pbase + kGradPerPhase * a.tpl.n_phases;
    for (int k = threadIdx.x; k < ng; k += blockDim.x) {
        const bool w = k < pbase ? want_leaf(a.want, k / kGradPerLeaf)
                     : k < sbase ? want_phase(a.want, (k - pbase) / kGradPerPhase)
                                 : want_scale(a.want, k - sbase);
        if (!w) gr[k] = 0.;
    }
}

template <typename T>
size_t adj_slab_bytes(int N) { return sizeof(Cx<T>) * (size_t)(N / 2 + 1) * N; }

// ROW_THREADS: one block-wide FFT per row pair; COL_THREADS: 512 where the block FFT allows
// it (N / R <= 2048), so that the reverse pass keeps 128 registers per thread, else 1024.
template <typename T, int ROW_THREADS, int COL_THREADS>
int launch_adj_large_t(const AdjArgs& args, int N, void* work, size_t work_bytes, cudaStream_t stream)
{
    const size_t slab = adj_slab_bytes<T>(N);
    if (!work || work_bytes < slab) return set_error(GSB_ERR_INVALID, "adjoint workspace too small");
    const size_t row_sm = sizeof(Cx<T>) * N;
    const size_t base = ((sizeof(AdjSmem) + 15) & ~size_t(15)) + sizeof(Cx<T>) * N;
    if (base + 1024 > kSmemLimit) return set_error(GSB_ERR_UNSUPPORTED, "FFT size too large for this precision");
    const size_t room = kSmemLimit - base - 1024;
    const int cache_bytes = int(std::min<size_t>(room, 160 * 1024) & ~size_t(15));
    const size_t col_sm = ((base + 15) & ~size_t(15)) + cache_bytes;
    const double2* tw = nullptr;
    int rc = fft_twiddles(N, stream, &tw);
    if (rc) return rc;
    const bool ii = has_image_leaves(args.tpl);
    GSB_CUDA_CHECK(cudaFuncSetAttribute(adj_large_row_kernel<T, ROW_THREADS>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(row_sm)));
    if (ii)
        GSB_CUDA_CHECK(cudaFuncSetAttribute(adj_large_col_kernel<T, COL_THREADS, true>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(col_sm)));
    else
        GSB_CUDA_CHECK(cudaFuncSetAttribute(adj_large_col_kernel<T, COL_THREADS, false>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(col_sm)));
    const int ng = grad_count(args.tpl);
    GSB_CUDA_CHECK(cudaMemsetAsync(args.grad, 0, sizeof(double) * (size_t)ng * args.n_stamps, stream));
    const int chunk = int(std::max<size_t>(1, std::min<size_t>(work_bytes / slab, 65535)));
    DeviceState* st = device_state();
    for (int s0 = 0; s0 < args.n_stamps; s0 += chunk) {
        const int n = std::min(chunk, args.n_stamps - s0);
        AdjLargeArgs la;
        la.a = args;
        la.a.n_stamps = n;
        la.a.leaves = args.leaves + (size_t)s0 * args.tpl.n_leaves;
        la.a.phases = args.phases ? args.phases + (size_t)s0 * args.tpl.n_phases : nullptr;
        la.a.scales = args.scales ? args.scales + (size_t)s0 * args.tpl.n_scales : nullptr;
        la.a.stamps = args.stamps + s0;
        la.a.grad = args.grad + (size_t)s0 * ng;
        la.N = N;
        la.tw = tw;
        la.W = work;
        la.cache_bytes = cache_bytes;
        const int gr = std::max(1, std::min(N / 2, (2 * st->sm_count + n - 1) / n));
        adj_large_row_kernel<T, ROW_THREADS><<<dim3(gr, n), ROW_THREADS, row_sm, stream>>>(la);
        GSB_CUDA_CHECK(cudaGetLastError());
        const int gx = std::max(1, std::min(N / 2 + 1, (2 * st->sm_count + n - 1) / n));
        if (ii) adj_large_col_kernel<T, COL_THREADS, true><<<dim3(gx, n), COL_THREADS, col_sm, stream>>>(la);
        else adj_large_col_kernel<T, COL_THREADS, false><<<dim3(gx, n), COL_THREADS, col_sm, stream>>>(la);
        GSB_CUDA_CHECK(cudaGetLastError());
    }
    adj_large_finalize_kernel<<<args.n_stamps, 128, 0, stream>>>(args);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

template <typename T>
int launch_adj_large(const AdjArgs& args, int N, void* work, size_t work_bytes, cudaStream_t stream)
{
    // the block FFT takes N / R <= 4 blockDim.x butterflies per pass (R = 3 for the first pass of
    // N = 3 * 2^a, else 4)
    const int first = (N % 3 == 0) ? N / 3 : N / 4;
    if (first <= 2048 && N / 4 <= 2048) return launch_adj_large_t<T, 1024, 512>(args, N, work, work_bytes, stream);
    return launch_adj_large_t<T, 1024, 1024>(args, N, work, work_bytes, stream);
}

}  // namespace

size_t adjoint_large_workspace_size(int N, int n_stamps, int precision)
{
    const size_t slab = precision == GSB_F64 ? adj_slab_bytes<double>(N) : adj_slab_bytes<float>(N);
    // up to 8 GiB of slabs per chunk, at least one stamp
    const size_t budget = size_t(8) << 30;
    return std::max<size_t>(1, std::min<size_t>((size_t)n_stamps, budget / slab)) * slab;
}

int adjoint_large(const AdjArgs& args, int N, int precision, size_t work_bytes, cudaStream_t stream)
{
    return precision == GSB_F64 ? launch_adj_large<double>(args, N, args.work, work_bytes, stream)
                                : launch_adj_large<float>(args, N, args.work, work_bytes, stream);
}

}  // namespace gsb
