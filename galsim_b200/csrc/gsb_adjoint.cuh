// Adjoint of the fused FFT draw (reverse mode), one CTA per stamp.
//
// The forward kernel computes, per stamp, image(x, y) = (1/N^2) sum_c w_c Re(sum_r X(c, r)
// e^{+2 pi i (c x + r y) / N}) over the Hermitian half plane c = 0..N/2 (w_c = 1 for c = 0 and
// N/2, else 2), where X is the wrapped k-image: the program summed over the aliases of (c, r)
// inside the Nk x Nk evaluation grid.  For a loss L with image cotangent G = dL/dimage,
//     dL = sum_{c,r} (w_c / N^2) Re(Ghat(c, r) dX(c, r)),
//     Ghat(c, r) = sum_pixels G(x, y) e^{+2 pi i (c x + r y) / N},
// i.e. Ghat is the forward-sign DFT of the zero-padded cotangent at the pixels' (x mod N,
// y mod N) positions.  The kernel computes Ghat with the same warp Stockham FFTs (rows in
// packed pairs, then columns), then visits every alias exactly as the forward gather does and
// runs the program in reverse at that k-point, accumulating
//   per leaf   d/dflux, d/dA, d/dB, d/dC, d/dD (its Jacobian), d/dn (Sersic index)
//   per phase  d/dcenx, d/dceny, d/dflux_scaling, d/dA..D (the phase's Jacobian)
//   per scale  d/dscale
// The k-grid is recomputed, never stored.
#pragma once

#include "gsb_draw.cuh"
#include "gsb_grad.cuh"

namespace gsb {

constexpr int kGradPerLeaf = 6;
constexpr int kGradPerPhase = 7;
constexpr int kMaxGrad = kGradPerLeaf * GSB_MAX_LEAVES + kGradPerPhase * GSB_MAX_PHASES + GSB_MAX_SCALES;

__host__ __device__ inline int grad_count(const gsb_template& tpl)
{
    return kGradPerLeaf * tpl.n_leaves + kGradPerPhase * tpl.n_phases + tpl.n_scales;
}

struct AdjArgs {
    gsb_template tpl;
    int n_stamps;
    const gsb_leaf* leaves;
    const gsb_phase* phases;
    const double* scales;
    const gsb_stamp* stamps;
    const double* sersic_header;
    const double4* sersic_node;
    const double* sersic_dheader;
    const double4* sersic_dnode;
    int sersic_stride;
    const void* cot;      // cotangent images, same layout as the forward output
    int cot_dtype;
    double* grad;         // n_stamps * grad_count(tpl)
    unsigned want;        // records whose gradients are wanted (leaf l: bit l, phase p: 8 + p, scale q: 16 + q)
    void* work;           // per-CTA W slabs when W does not fit in shared memory
};

// Atoms of the factored adjoint held in registers.
constexpr int kAdjAtoms = 3;

struct AdjSmem {
    StampSmem S;
    SersicDnView dn[GSB_MAX_LEAVES];
    int child1[GSB_MAX_OPS];
    int child2[GSB_MAX_OPS];
    double gacc[kMaxGrad];
};

// Operand op indices of every op of the postfix program (thread 0).
__device__ inline void program_children(const gsb_template& tpl, int* c1, int* c2)
{
    int st[GSB_MAX_OPS];
    int sp = 0;
    for (int o = 0; o < tpl.n_ops; ++o) {
        const int code = tpl.op_code[o];
        c1[o] = c2[o] = -1;
        if (code == GSB_OP_LEAF) {
            st[sp++] = o;
        } else if (code == GSB_OP_MUL || code == GSB_OP_ADD) {
            c2[o] = st[--sp];
            c1[o] = st[sp - 1];
            st[sp - 1] = o;
        } else {
            c1[o] = st[sp - 1];
            st[sp - 1] = o;
        }
    }
}

// Reverse-mode pass of the ops [o0, o1) (a complete subtree, or the whole program) at k index
// (i, j) with output cotangent u (contribution Re(u * dF)); gradients are added into acc.
template <typename T, bool II = true>
__device__ __noinline__ void adjoint_range(const gsb_template& tpl, const AdjSmem& A, double dk, int i,
                                           int j, const GridRef& g, Cx<T> u, T* acc, int o0, int o1)
{
    const StampSmem& S = A.S;
    Cx<T> val[GSB_MAX_OPS];
    Cx<T> adj[GSB_MAX_OPS];
    LeafD<T> ld[GSB_MAX_LEAVES];
    Cx<T> pe[GSB_MAX_PHASES];
    const T kx = T(i) * T(dk), ky = T(j) * T(dk);
    const int n_ops = o1;
    for (int o = o0; o < n_ops; ++o) {
        const int code = tpl.op_code[o], arg = tpl.op_arg[o];
        const int a = A.child1[o], b = A.child2[o];
        if (code == GSB_OP_LEAF) {
            if (II && S.leaf[arg].type == GSB_INTERPOLATED) {
                // an image leaf enters with its complex value and no gradient entries of its own
                ld[arg] = LeafD<T>{T(0), T(0), T(0), T(0), T(0)};
                val[o] = ii_kvalue<T>(S.leaf[arg], dk, i, j);
            } else {
                ld[arg] = leaf_grad<T>(S.leaf[arg], S.sersic, A.dn, kx, ky, g, i - g.x0, j - g.y0);
                val[o] = cx<T>(ld[arg].v, T(0));
            }
        } else if (code == GSB_OP_MUL) {
            val[o] = cmul<T>(val[a], val[b]);
        } else if (code == GSB_OP_ADD) {
            val[o] = cadd<T>(val[a], val[b]);
        } else if (code == GSB_OP_PHASE) {
            double tt = i * S.phase_ax[arg] + j * S.phase_ay[arg];
            tt -= rint(tt);
            T sn, cs;
            sincospi(T(-2. * tt), &sn, &cs);
            pe[arg] = cx<T>(cs, sn);
            val[o] = cscale<T>(cmul<T>(val[a], pe[arg]), T(S.phase[arg].flux_scaling));
        } else {
            val[o] = cscale<T>(val[a], T(S.scale[arg]));
        }
        adj[o] = cx<T>(T(0), T(0));
    }
    adj[n_ops - 1] = u;
    const int pbase = kGradPerLeaf * tpl.n_leaves;
    const int sbase = pbase + kGradPerPhase * tpl.n_phases;
    for (int o = n_ops - 1; o >= o0; --o) {
        const int code = tpl.op_code[o], arg = tpl.op_arg[o];
        const int a = A.child1[o], b = A.child2[o];
        const Cx<T> w = adj[o];
        if (code == GSB_OP_LEAF) {
            const LeafD<T>& d = ld[arg];
            const T ar = w.x;
            T* gl = acc + kGradPerLeaf * arg;
            gl[0] += ar * d.unit;
            gl[1] += ar * d.gx * kx;
            gl[2] += ar * d.gy * kx;
            gl[3] += ar * d.gx * ky;
            gl[4] += ar * d.gy * ky;
            gl[5] += ar * d.gn;
        } else if (code == GSB_OP_MUL) {
            adj[a] = cadd<T>(adj[a], cmul<T>(w, val[b]));
            adj[b] = cadd<T>(adj[b], cmul<T>(w, val[a]));
        } else if (code == GSB_OP_ADD) {
            adj[a] = cadd<T>(adj[a], w);
            adj[b] = cadd<T>(adj[b], w);
        } else if (code == GSB_OP_PHASE) {
            const gsb_phase& P = S.phase[arg];
            const T fs = T(P.flux_scaling);
            const Cx<T> e = pe[arg];
            adj[a] = cadd<T>(adj[a], cscale<T>(cmul<T>(w, e), fs));
            const Cx<T> we = cmul<T>(cmul<T>(w, val[a]), e);
            const T z = fs * we.y;                   // dL/dtheta with f = fs exp(-i theta)
            const T cxp = T(P.cenx), cyp = T(P.ceny);
            T* gp = acc + pbase + kGradPerPhase * arg;
            gp[0] += z * (T(P.jac[0]) * kx + T(P.jac[2]) * ky);
            gp[1] += z * (T(P.jac[1]) * kx + T(P.jac[3]) * ky);
            gp[2] += we.x;
            gp[3] += z * kx * cxp;
            gp[4] += z * kx * cyp;
            gp[5] += z * ky * cxp;
            gp[6] += z * ky * cyp;
        } else {
            adj[a] = cadd<T>(adj[a], cscale<T>(w, T(S.scale[arg])));
            acc[sbase + arg] += cmul<T>(w, val[a]).x;
        }
    }
}

// Gradients of the leaves of a Sum atom (LEAF and ADD ops [o0, o1)) with cotangent w: each
// leaf receives w unchanged.
template <typename T>
__device__ __noinline__ void sum_atom_grads(const gsb_template& tpl, const AdjSmem& A, unsigned want,
                                            T kx, T ky, int i, int j, const GridRef& g, Cx<T> w, T* acc,
                                            int o0, int o1)
{
    const T ar = w.x;
    for (int o = o0; o < o1; ++o) {
        if (tpl.op_code[o] != GSB_OP_LEAF) continue;
        const int l = tpl.op_arg[o];
        if (!want_leaf(want, l)) continue;
        const LeafD<T> d = leaf_grad<T>(A.S.leaf[l], A.S.sersic, A.dn, kx, ky, g, i - g.x0, j - g.y0);
        T* gl = acc + kGradPerLeaf * l;
        gl[0] += ar * d.unit;
        gl[1] += ar * d.gx * kx;
        gl[2] += ar * d.gy * kx;
        gl[3] += ar * d.gx * ky;
        gl[4] += ar * d.gy * ky;
        gl[5] += ar * d.gn;
    }
}

// Factored reverse pass at (i, j): F = prod_a atom_a * XS[i] YS[j]; the cotangent of atom a
// is u XS YS prod_{b != a} atom_b (prefix and suffix products, no division).  Leaf, phase and
// scale atoms accumulate into ga[a][*] (registers); subtree atoms run adjoint_range into acc.
template <typename T, bool II = true>
__device__ __forceinline__ void adjoint_point_factored(const gsb_template& tpl, const AdjSmem& A,
                                                       const unsigned char* cache, unsigned want, double dk,
                                                       int i, int j, const GridRef& g, Cx<T> u,
                                                       T (&ga)[kAdjAtoms][kGradPerPhase], T* acc)
{
    const StampSmem& S = A.S;
    const int hk = g.n / 2;
    const T kx = T(i) * T(dk), ky = T(j) * T(dk);
    const int na = S.n_atoms;
    // ld[a] holds a leaf atom's derivatives, or a phase atom's unit phasor in (gx, gy)
    Cx<T> val[kAdjAtoms], pre[kAdjAtoms];
    LeafD<T> ld[kAdjAtoms];
    Cx<T> run = cx<T>(T(1), T(0));
#pragma unroll
    for (int a = 0; a < kAdjAtoms; ++a) {
        val[a] = cx<T>(T(1), T(0));
        ld[a] = LeafD<T>{T(0), T(0), T(0), T(0), T(0)};
        if (a < na) {
            const int kind = S.atom_kind[a];
            const int o0 = S.atom_o0[a], o1 = S.atom_o1[a];
            if (kind == kAtomPhase) {
                const int p = S.atom_arg[a];
                double tt = i * S.phase_ax[p] + j * S.phase_ay[p];
                tt -= rint(tt);
                T sn, cs;
                sincospi(T(-2. * tt), &sn, &cs);
                ld[a].gx = cs;
                ld[a].gy = sn;
                val[a] = cscale<T>(cx<T>(cs, sn), T(S.phase[p].flux_scaling));
            } else if (kind == kAtomScale) {
                val[a] = cx<T>(T(S.scale[S.atom_arg[a]]), T(0));
            } else if (o1 - o0 == 1) {
                const int l = tpl.op_arg[o0];
                if (want_leaf(want, l) && !(II && S.leaf[l].type == GSB_INTERPOLATED)) {
                    ld[a] = leaf_grad<T>(S.leaf[l], S.sersic, A.dn, kx, ky, g, i - g.x0, j - g.y0);
                    val[a] = cx<T>(ld[a].v, T(0));
                } else {
                    val[a] = leaf_cfast<T, II>(S, cache, l, kx, ky, i, j, g);
                }
            } else {
                val[a] = eval_range<T, II>(tpl, S, cache, dk, i, j, g, o0, o1);
            }
        }
        pre[a] = run;
        run = cmul<T>(run, val[a]);
    }
    const Cx<T>* XS = reinterpret_cast<const Cx<T>*>(cache + S.xy_cache);
    const Cx<T> us = cmul<T>(u, cmul<T>(XS[i], XS[hk + 1 + j + hk]));
    Cx<T> suf = cx<T>(T(1), T(0));
#pragma unroll
    for (int a = kAdjAtoms - 1; a >= 0; --a) {
        if (a < na) {
            const Cx<T> w = cmul<T>(cmul<T>(us, pre[a]), suf);
            const int kind = S.atom_kind[a];
            const int o0 = S.atom_o0[a], o1 = S.atom_o1[a];
            if (kind == kAtomPhase) {
                const gsb_phase& P = S.phase[S.atom_arg[a]];
                const Cx<T> we = cmul<T>(w, cx<T>(ld[a].gx, ld[a].gy));
                const T z = T(P.flux_scaling) * we.y;
                const T cxp = T(P.cenx), cyp = T(P.ceny);
                ga[a][0] += z * (T(P.jac[0]) * kx + T(P.jac[2]) * ky);
                ga[a][1] += z * (T(P.jac[1]) * kx + T(P.jac[3]) * ky);
                ga[a][2] += we.x;
                ga[a][3] += z * kx * cxp;
                ga[a][4] += z * kx * cyp;
                ga[a][5] += z * ky * cxp;
                ga[a][6] += z * ky * cyp;
            } else if (kind == kAtomScale) {
                ga[a][0] += w.x;
            } else if (o1 - o0 == 1) {
                const T ar = w.x;
                ga[a][0] += ar * ld[a].unit;
                ga[a][1] += ar * ld[a].gx * kx;
                ga[a][2] += ar * ld[a].gy * kx;
                ga[a][3] += ar * ld[a].gx * ky;
                ga[a][4] += ar * ld[a].gy * ky;
                ga[a][5] += ar * ld[a].gn;
            } else if (kind == kAtomSum) {
                sum_atom_grads<T>(tpl, A, want, kx, ky, i, j, g, w, acc, o0, o1);
            } else {
                adjoint_range<T, II>(tpl, A, dk, i, j, g, w, acc, o0, o1);
            }
            suf = cmul<T>(suf, val[a]);
        }
    }
}

template <typename T>
__device__ inline T load_cot(const void* p, int dtype, long long idx)
{
    return dtype == GSB_F32 ? T(reinterpret_cast<const float*>(p)[idx])
                            : T(reinterpret_cast<const double*>(p)[idx]);
}

// Warps per CTA: 16, or 8 where 16 FFT buffers of N complex T do not fit (double, N >= 768).
template <typename T, int N>
__host__ __device__ constexpr int adj_warps()
{
    return ((sizeof(AdjSmem) + 15) / 16 * 16 + sizeof(Cx<T>) * N * (1 + kWarps) + kCacheBytes + 4096 <=
            kSmemLimit) ? kWarps : kWarps / 2;
}

template <typename T, int N, bool WSMEM, bool II>
__global__ void __launch_bounds__(adj_warps<T, N>() * 32) adjoint_fused_kernel(const __grid_constant__ AdjArgs a)
{
    constexpr int NW = adj_warps<T, N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int H = N / 2 + 1;
    constexpr int WS = N + 1;
    AdjSmem& A = *reinterpret_cast<AdjSmem*>(smem_raw);
    StampSmem& S = A.S;
    size_t off = (sizeof(AdjSmem) + 15) & ~size_t(15);
    Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw + off);
    off += sizeof(Cx<T>) * N;
    Cx<T>* scratch = reinterpret_cast<Cx<T>*>(smem_raw + off);
    off += sizeof(Cx<T>) * N * NW;
    Cx<T>* W = WSMEM ? reinterpret_cast<Cx<T>*>(smem_raw + off)
                     : reinterpret_cast<Cx<T>*>(a.work) + (size_t)blockIdx.x * H * WS;
    if (WSMEM) off += sizeof(Cx<T>) * H * WS;
    unsigned char* cache = smem_raw + ((off + 15) & ~size_t(15));

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Cx<T>* buf = scratch + warp * N;
    fill_twiddles<T>(tw, N);
    const double dk = 2. * kPi / N;
    const T inv_n2 = T(1) / (T(N) * T(N));
    const int ng = grad_count(a.tpl);
    if (threadIdx.x == 0) program_children(a.tpl, A.child1, A.child2);

    for (int s = blockIdx.x; s < a.n_stamps; s += gridDim.x) {
        __syncthreads();
        load_stamp(S, a.tpl, s, a.leaves, a.phases, a.scales, a.stamps, a.sersic_header,
                   a.sersic_node, a.sersic_stride, 1. / N);
        if (threadIdx.x < a.tpl.n_leaves && S.leaf[threadIdx.x].type == GSB_SERSIC && a.sersic_dheader) {
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
        const int Nk = G.Nk;
        const int hk = Nk / 2;
        const GridRef g{dk, 0, -hk, hk + 1, Nk + 1};
        if (threadIdx.x == 0) plan_caches<T, II>(S, a.tpl, Nk, a.want);
        __syncthreads();
        fill_caches<T, II>(S, a.tpl, cache, dk, Nk);
        __syncthreads();
        const bool factored = S.xy_cache >= 0 && S.n_atoms <= kAdjAtoms;
        bool subtree = !factored;
        if (factored)
            for (int t = 0; t < S.n_atoms; ++t)
                subtree |= (S.atom_kind[t] == kAtomRange || S.atom_kind[t] == kAtomSum) &&
                           S.atom_o1[t] - S.atom_o0[t] > 1;

        // ---- row phase: forward-sign DFT of pairs of cotangent rows ----
        const int npairs = (G.ny + 1) / 2;
        for (int p = warp; p < npairs; p += NW) {
            const bool two = 2 * p + 1 < G.ny;
            for (int x = lane; x < N; x += 32) buf[x] = cx<T>(T(0), T(0));
            __syncwarp();
            const long long row1 = G.out_offset + (long long)(2 * p) * G.nx;
            for (int i = lane; i < G.nx; i += 32) {
                const T g1 = load_cot<T>(a.cot, a.cot_dtype, row1 + i);
                const T g2 = two ? load_cot<T>(a.cot, a.cot_dtype, row1 + G.nx + i) : T(0);
                buf[pmod(G.xmin + i, N)] = cx<T>(g1, g2);
            }
            __syncwarp();
            warp_fft<T, N, +1>(buf, tw);
            const int y1 = pmod(G.ymin + 2 * p, N), y2 = pmod(G.ymin + 2 * p + 1, N);
            for (int c = lane; c < H; c += 32) {
                const Cx<T> z = buf[c];
                const Cx<T> zm = buf[c == 0 ? 0 : N - c];
                W[(size_t)c * WS + y1] = cx<T>(T(0.5) * (z.x + zm.x), T(0.5) * (z.y - zm.y));
                if (two) W[(size_t)c * WS + y2] = cx<T>(T(0.5) * (z.y + zm.y), T(0.5) * (zm.x - z.x));
            }
            __syncwarp();
        }
        __syncthreads();

        // ---- column phase: forward-sign DFT along y, then the reverse pass per alias ----
        // Each lane accumulates its gradient terms over all of its warp's columns; the warp
        // reduces them once per stamp.
        T acc[kMaxGrad];
        T ga[kAdjAtoms][kGradPerPhase];
        if (subtree)
            for (int k = 0; k < ng; ++k) acc[k] = T(0);
#pragma unroll
        for (int t = 0; t < kAdjAtoms; ++t)
#pragma unroll
            for (int e = 0; e < kGradPerPhase; ++e) ga[t][e] = T(0);
        for (int c = warp; c < H; c += NW) {
            for (int y = lane; y < N; y += 32)
                buf[y] = pmod(y - G.ymin, N) < G.ny ? W[(size_t)c * WS + y] : cx<T>(T(0), T(0));
            __syncwarp();
            warp_fft<T, N, +1>(buf, tw);
            const T wc = (c == 0 || 2 * c == N) ? inv_n2 : T(2) * inv_n2;
            const int alo = ceil_div(-hk - c, N), ahi = floor_div(hk - c, N);
            for (int r = lane; r < N; r += 32) {
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
            __syncwarp();
        }
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
        // Sersic leaves given by half-light radius: r0 = hlr / r_e(n), so at fixed hlr
        // d/dn picks up -d ln r_e/dn * d/d ln r0, and d/d ln r0 = sum_ij J_ij d/dJ_ij.
        if (threadIdx.x < a.tpl.n_leaves && want_leaf(a.want, threadIdx.x)) {
            const LeafParams& L = S.leaf[threadIdx.x];
            if (L.type == GSB_SERSIC && (L.flags & GSB_LEAF_SIZE_IS_HLR)) {
                double* gl = A.gacc + kGradPerLeaf * threadIdx.x;
                const double glnr0 = L.jac[0] * gl[1] + L.jac[1] * gl[2] + L.jac[2] * gl[3] + L.jac[3] * gl[4];
                gl[5] -= A.dn[threadIdx.x].dlnre * glnr0;
            }
        }
        __syncthreads();
        // entries of records outside the want mask are written as zero
        const int pbase = kGradPerLeaf * a.tpl.n_leaves;
        const int sbase = pbase + kGradPerPhase * a.tpl.n_phases;
        for (int k = threadIdx.x; k < ng; k += blockDim.x) {
            const bool w = k < pbase ? want_leaf(a.want, k / kGradPerLeaf)
                         : k < sbase ? want_phase(a.want, (k - pbase) / kGradPerPhase)
                                     : want_scale(a.want, k - sbase);
            a.grad[(size_t)s * ng + k] = w ? A.gacc[k] : 0.;
        }
    }
}

template <typename T, int N>
constexpr size_t adj_smem_bytes(bool wsmem)
{
    size_t off = (sizeof(AdjSmem) + 15) & ~size_t(15);
    off += sizeof(Cx<T>) * N * (1 + adj_warps<T, N>());
    if (wsmem) off += sizeof(Cx<T>) * (N / 2 + 1) * (N + 1);
    return ((off + 15) & ~size_t(15)) + kCacheBytes;
}

template <typename T, int N>
constexpr bool adj_w_fits_smem()
{
    return adj_smem_bytes<T, N>(true) <= kSmemLimit;
}

template <typename T, int N>
int adj_grid(int n_stamps)
{
    DeviceState* st = device_state();
    const size_t sm = adj_smem_bytes<T, N>(adj_w_fits_smem<T, N>());
    int per_sm = int(std::min<size_t>(kSmemLimit / sm, 4));
    if (per_sm < 1) per_sm = 1;
    return std::max(1, std::min(n_stamps, st->sm_count * per_sm));
}

template <typename T, int N>
size_t adj_workspace_bytes_for(int n_stamps)
{
    if (adj_w_fits_smem<T, N>()) return 0;
    return sizeof(Cx<T>) * (size_t)(N / 2 + 1) * (N + 1) * adj_grid<T, N>(n_stamps);
}

template <typename T, int N>
int launch_adjoint(const AdjArgs& args, size_t work_bytes, cudaStream_t stream)
{
    constexpr bool wsmem = adj_w_fits_smem<T, N>();
    constexpr size_t sm = adj_smem_bytes<T, N>(wsmem);
    const int grid = adj_grid<T, N>(args.n_stamps);
    if (!wsmem && (args.work == nullptr || work_bytes < adj_workspace_bytes_for<T, N>(args.n_stamps)))
        return set_error(GSB_ERR_INVALID, "adjoint workspace too small");
    // programs without image leaves run the instance compiled without their code
    if (has_image_leaves(args.tpl)) {
        GSB_CUDA_CHECK(cudaFuncSetAttribute(adjoint_fused_kernel<T, N, wsmem, true>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        adjoint_fused_kernel<T, N, wsmem, true><<<grid, adj_warps<T, N>() * 32, sm, stream>>>(args);
    } else {
        GSB_CUDA_CHECK(cudaFuncSetAttribute(adjoint_fused_kernel<T, N, wsmem, false>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        adjoint_fused_kernel<T, N, wsmem, false><<<grid, adj_warps<T, N>() * 32, sm, stream>>>(args);
    }
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

}  // namespace gsb
