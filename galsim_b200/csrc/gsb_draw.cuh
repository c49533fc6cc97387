// Fused FFT drawing kernels.
//
// draw_fused_kernel<T, N, W_IN_SMEM>: one CTA draws one stamp at a time (persistent loop over
// the stamps of an FFT-size bucket):
//   1. column phase: each warp takes columns kx = 0..N/2 of the wrapped k-image; every lane
//      builds the wrapped value of its rows by summing the program over all aliases
//      (kx + a N, ky + b N) inside the Nk x Nk evaluation grid -- the Hermitian wrap of
//      wrapImage(hermx=True) (src/Image.cpp:578-727) done as a gather -- then the warp
//      inverse-transforms the column (length N) and stores it into W (shared memory, or a
//      per-CTA global slab when it does not fit);
//   2. row phase: each warp packs two needed image rows as one complex row
//      (row1 + i row2, each Hermitian-extended in kx), inverse-transforms it and writes the
//      pixels that fall inside the stamp, scaled by 1/N^2, with the compensated flux sum.
// This is drawFFT (gsobject.py:2014-2045) = drawFFT_makeKImage + _drawKImage + wrap +
// irfft(shift_in, shift_out) (src/Image.cpp:815-912) + drawFFT_finish, with no k-image in
// HBM.  The output pixel (px, py) is the inverse DFT at (px mod N, py mod N), which is what
// irfft's half swap and (-1)^(i+j) pre-multiplication produce.
#pragma once
#include <algorithm>
#include <string>

#include "gsb_fft.cuh"
#include "gsb_internal.cuh"
#include "gsb_interp.cuh"
#include "gsb_profiles.cuh"

namespace gsb {


constexpr int kWarps = 16;          // warps per CTA (fewer where their FFT scratch does not fit)

struct StampSmem {
    LeafParams leaf[GSB_MAX_LEAVES];
    SersicTableView sersic[GSB_MAX_LEAVES];
    gsb_phase phase[GSB_MAX_PHASES];
    double phase_ax[GSB_MAX_PHASES];   // phase turns per k index, x and y
    double phase_ay[GSB_MAX_PHASES];
    double scale[GSB_MAX_SCALES];
    gsb_stamp geom;
    double flux_part[kWarps];
    // Per-stamp shared-memory caches (offsets in bytes into the cache area, -1 = not cached):
    // separable leaf factors X[i], Y[j + Nk/2]; phase factors PX[i], PY[j + Nk/2]; Sersic nodes.
    int leaf_cache[GSB_MAX_LEAVES];
    int phase_cache[GSB_MAX_PHASES];
    int sersic_cache[GSB_MAX_LEAVES];
    int ii_cache[GSB_MAX_LEAVES];      // InterpolatedImage taps per column / row (IITaps)
    int regstack;      // the program fits the 4-deep register stack
    // Factored form of the program (see plan_factored): the root is a product of atoms; the
    // separable atoms (diagonal Box / Gaussian leaves, phases, scales) are folded into
    // XS[i] YS[j + Nk/2] (complex, at offset xy_cache, -1 = not factored) and the others are
    // evaluated per k-point over their postfix op ranges [atom_o0, atom_o1).
    int xy_cache;
    int n_atoms;
    short atom_o0[GSB_MAX_OPS];
    short atom_o1[GSB_MAX_OPS];
    unsigned char atom_kind[GSB_MAX_OPS];      // kAtomRange, kAtomPhase (arg), kAtomScale (arg)
    unsigned char atom_arg[GSB_MAX_OPS];
    unsigned char leaf_sep[GSB_MAX_LEAVES];    // leaf folded into XS / YS
    unsigned char phase_sep[GSB_MAX_PHASES];   // phase folded into XS / YS
    unsigned char scale_sep[GSB_MAX_SCALES];   // scale folded into XS / YS
};

// Bytes of shared memory reserved for the per-stamp caches.
constexpr int kCacheBytes = 24 * 1024;

constexpr size_t kSmemLimit = 227 * 1024;

// Warps per CTA of the fused kernels for (T, N): 16, or 8 where 16 per-warp FFT buffers of N
// complex T (plus twiddles, stamp state and caches) exceed the 227 KB of shared memory
// (double at N >= 768).
template <typename T, int N>
__host__ __device__ constexpr int fused_warps()
{
    return ((sizeof(StampSmem) + 15) / 16 * 16 + sizeof(Cx<T>) * N * (1 + kWarps) + kCacheBytes + 4096 <=
            kSmemLimit) ? kWarps : kWarps / 2;
}

struct DrawArgs {
    gsb_template tpl;
    int n_stamps;
    const gsb_leaf* leaves;
    const gsb_phase* phases;
    const double* scales;
    const gsb_stamp* stamps;
    const double* sersic_header;
    const double4* sersic_node;
    int sersic_stride;
    void* out;
    int out_dtype;
    int add;
    double* added_flux;
    void* work;          // per-CTA W slabs when W does not fit in shared memory
};

__device__ inline int floor_div(int a, int n) { return a >= 0 ? a / n : -((-a + n - 1) / n); }
__device__ inline int ceil_div(int a, int n) { return -floor_div(-a, n); }
__device__ inline int pmod(int a, int n) { const int r = a % n; return r < 0 ? r + n : r; }

// Load stamp s's leaves / phases / scales into shared memory.
__device__ inline void load_stamp(StampSmem& S, const gsb_template& tpl, int s, const gsb_leaf* leaves,
                           const gsb_phase* phases, const double* scales, const gsb_stamp* stamps,
                           const double* sh, const double4* snode, int sstride, double dk_over_2pi)
{
    const int t = threadIdx.x;
    if (t < tpl.n_leaves) {
        const gsb_leaf& g = leaves[(size_t)s * tpl.n_leaves + t];
        LeafParams& L = S.leaf[t];
        for (int i = 0; i < 4; ++i) L.jac[i] = g.jac[i];
        L.flux = g.flux;
        for (int i = 0; i < 8; ++i) L.d[i] = g.d[i];
        L.flags = g.flags;
        L.type = tpl.leaf_type[t];
        L.table = t;
        if (L.type == GSB_SERSIC && sh) {
            const double* H = sh + (size_t)g.table * kSersicHeader;
            SersicTableView& v = S.sersic[t];
            v.n = int(H[kSH_NUSED]);
            v.front = H[kSH_FRONT];
            v.da = H[kSH_DA];
            v.ksq_min = H[kSH_KSQMIN];
            v.ksq_max = H[kSH_KSQMAX];
            v.kderiv2 = H[kSH_KD2];
            v.kderiv4 = H[kSH_KD4];
            v.highk_a = H[kSH_HIGHA];
            v.highk_b = H[kSH_HIGHB];
            v.node = snode + (size_t)g.table * sstride;
        }
    }
    if (t >= 32 && t < 32 + tpl.n_phases) {
        const int i = t - 32;
        const gsb_phase& P = phases[(size_t)s * tpl.n_phases + i];
        S.phase[i] = P;
        // exp(-i (kx' cx + ky' cy)) with k' = jac^T k and k = (i, j) dk:
        // argument = 2 pi (i ax + j ay), ax = (A cx + B cy) dk / 2 pi, ay = (C cx + D cy) dk / 2 pi
        S.phase_ax[i] = (P.jac[0] * P.cenx + P.jac[1] * P.ceny) * dk_over_2pi;
        S.phase_ay[i] = (P.jac[2] * P.cenx + P.jac[3] * P.ceny) * dk_over_2pi;
    }
    if (t >= 64 && t < 64 + tpl.n_scales) S.scale[t - 64] = scales[(size_t)s * tpl.n_scales + (t - 64)];
    if (t == 96 && stamps) S.geom = stamps[s];
}

// Evaluate the program at k index (i, j) (kx = i dk, ky = j dk) of grid g.
// II: the program may hold InterpolatedImage leaves (their code is compiled in only then).
template <typename T, bool II = true>
__device__ __noinline__ Cx<T> eval_program(const gsb_template& tpl, const StampSmem& S, double dk, int i, int j,
                              const GridRef& g)
{
    Cx<T> stack[GSB_MAX_OPS];
    int sp = 0;
    const T kx = T(i * dk), ky = T(j * dk);
    const int gi = i - g.x0, gj = j - g.y0;
    for (int o = 0; o < tpl.n_ops; ++o) {
        const int code = tpl.op_code[o], arg = tpl.op_arg[o];
        if (code == GSB_OP_LEAF) {
            if (II && S.leaf[arg].type == GSB_INTERPOLATED)
                stack[sp++] = ii_kvalue<T>(S.leaf[arg], dk, i, j);
            else
                stack[sp++] = cx<T>(leaf_kvalue<T>(S.leaf[arg], S.sersic, kx, ky, g, gi, gj), T(0));
        } else if (code == GSB_OP_MUL) {
            --sp;
            stack[sp - 1] = cmul<T>(stack[sp - 1], stack[sp]);
        } else if (code == GSB_OP_ADD) {
            --sp;
            stack[sp - 1] = cadd<T>(stack[sp - 1], stack[sp]);
        } else if (code == GSB_OP_PHASE) {
            double tt = i * S.phase_ax[arg] + j * S.phase_ay[arg];
            tt -= rint(tt);
            T sn, cs;
            sincospi(T(-2. * tt), &sn, &cs);
            const T fs = T(S.phase[arg].flux_scaling);
            stack[sp - 1] = cmul<T>(stack[sp - 1], cx<T>(fs * cs, fs * sn));
        } else if (code == GSB_OP_SCALE) {
            stack[sp - 1] = cscale<T>(stack[sp - 1], T(S.scale[arg]));
        }
    }
    return stack[0];
}

template <typename T> struct NodeT;
template <> struct NodeT<float> { using type = float4; };
template <> struct NodeT<double> { using type = double4; };

// Decide which factors of this stamp are cached in shared memory (thread 0), in order:
// Sersic spline nodes, phase factors, separable leaf factors, until the budget is used.
// kAtomSum: a subtree of LEAF and ADD ops only (e.g. bulge + disk), whose cotangent passes
// unchanged to each of its leaves.
enum { kAtomRange = 0, kAtomPhase = 1, kAtomScale = 2, kAtomSum = 3 };

// want bits: leaf l = bit l, phase p = bit 8 + p, scale q = bit 16 + q.
__device__ __forceinline__ bool want_leaf(unsigned want, int l) { return (want >> l) & 1u; }
__device__ __forceinline__ bool want_phase(unsigned want, int p) { return (want >> (8 + p)) & 1u; }
__device__ __forceinline__ bool want_scale(unsigned want, int q) { return (want >> (16 + q)) & 1u; }

// Split the program's root product into atoms (thread 0).  MUL nodes are flattened; PHASE and
// SCALE nodes contribute a separable factor and pass their child on; a LEAF is separable when
// its value is X(i) Y(j) (Box or Gaussian with a diagonal Jacobian: the reference's 1-d fill);
// every other LEAF and every ADD subtree is an atom evaluated per point.  Factors named in
// `want` (the adjoint's differentiated records) are not folded: a wanted separable leaf stays a
// leaf atom, a wanted phase or scale becomes an atom of its own.  Returns false when the atoms
// do not fit the fixed arrays (the program is then evaluated unfactored).
__device__ inline bool plan_factored(StampSmem& S, const gsb_template& tpl, unsigned want = 0u)
{
    short c1[GSB_MAX_OPS], c2[GSB_MAX_OPS], start[GSB_MAX_OPS];
    short st[GSB_MAX_OPS];
    int sp = 0;
    for (int o = 0; o < tpl.n_ops; ++o) {
        const int code = tpl.op_code[o];
        c1[o] = c2[o] = -1;
        if (code == GSB_OP_LEAF) {
            start[o] = o;
            st[sp++] = o;
        } else if (code == GSB_OP_MUL || code == GSB_OP_ADD) {
            c2[o] = st[--sp];
            c1[o] = st[sp - 1];
            start[o] = start[c1[o]];
            st[sp - 1] = o;
        } else {
            c1[o] = st[sp - 1];
            start[o] = start[c1[o]];
            st[sp - 1] = o;
        }
    }
    for (int l = 0; l < GSB_MAX_LEAVES; ++l) S.leaf_sep[l] = 0;
    for (int p = 0; p < GSB_MAX_PHASES; ++p) S.phase_sep[p] = 0;
    for (int q = 0; q < GSB_MAX_SCALES; ++q) S.scale_sep[q] = 0;
    S.n_atoms = 0;
    sp = 0;
    st[sp++] = tpl.n_ops - 1;
    while (sp > 0) {
        const int o = st[--sp];
        const int code = tpl.op_code[o], arg = tpl.op_arg[o];
        if (code == GSB_OP_MUL) {
            st[sp++] = c1[o];
            st[sp++] = c2[o];
        } else if (code == GSB_OP_PHASE || code == GSB_OP_SCALE) {
            const bool ph = code == GSB_OP_PHASE;
            if (ph ? want_phase(want, arg) : want_scale(want, arg)) {
                S.atom_o0[S.n_atoms] = o;
                S.atom_o1[S.n_atoms] = o + 1;
                S.atom_kind[S.n_atoms] = ph ? kAtomPhase : kAtomScale;
                S.atom_arg[S.n_atoms] = (unsigned char)arg;
                ++S.n_atoms;
            } else if (ph) {
                S.phase_sep[arg] = 1;
            } else {
                S.scale_sep[arg] = 1;
            }
            st[sp++] = c1[o];
        } else {
            if (code == GSB_OP_LEAF && !want_leaf(want, arg)) {
                const LeafParams& L = S.leaf[arg];
                if ((L.type == GSB_BOX || L.type == GSB_GAUSSIAN) && !(L.flags & GSB_LEAF_JAC_GENERAL)) {
                    S.leaf_sep[arg] = 1;
                    continue;
                }
            }
            bool sum = code == GSB_OP_ADD;
            for (int q = start[o]; q <= o && sum; ++q)
                sum = tpl.op_code[q] == GSB_OP_LEAF || tpl.op_code[q] == GSB_OP_ADD;
            S.atom_o0[S.n_atoms] = start[o];
            S.atom_o1[S.n_atoms] = o + 1;
            S.atom_kind[S.n_atoms] = sum ? kAtomSum : kAtomRange;
            S.atom_arg[S.n_atoms] = (unsigned char)(code == GSB_OP_LEAF ? arg : 0);
            ++S.n_atoms;
        }
    }
    return true;
}

template <typename T, bool II = true>
__device__ inline void plan_caches(StampSmem& S, const gsb_template& tpl, int Nk, unsigned want = 0u,
                                   int budget = kCacheBytes)
{
    const int hk = Nk / 2;
    int used = 0;
    int depth = 0, maxd = 0;
    for (int o = 0; o < tpl.n_ops; ++o) {
        const int c = tpl.op_code[o];
        if (c == GSB_OP_LEAF) ++depth;
        else if (c == GSB_OP_MUL || c == GSB_OP_ADD) --depth;
        maxd = depth > maxd ? depth : maxd;
    }
    S.regstack = maxd <= 4;
    S.xy_cache = -1;
    {
        const int bytes = ((hk + 1 + Nk + 1) * (int)sizeof(Cx<T>) + 15) & ~15;
        if (S.regstack && bytes <= budget && plan_factored(S, tpl, want)) {
            S.xy_cache = used;
            used += bytes;
        } else {
            for (int l = 0; l < GSB_MAX_LEAVES; ++l) S.leaf_sep[l] = 0;
            for (int p = 0; p < GSB_MAX_PHASES; ++p) S.phase_sep[p] = 0;
            for (int q = 0; q < GSB_MAX_SCALES; ++q) S.scale_sep[q] = 0;
        }
    }
    for (int l = 0; l < tpl.n_leaves; ++l) {
        S.sersic_cache[l] = -1;
        S.leaf_cache[l] = -1;
        if (S.leaf[l].type == GSB_SERSIC) {
            const int bytes = (S.sersic[l].n * (int)sizeof(typename NodeT<T>::type) + 15) & ~15;
            if (used + bytes <= budget) { S.sersic_cache[l] = used; used += bytes; }
        }
    }
    // InterpolatedImage leaves with a diagonal Jacobian: the taps, weights and transform
    // factor of every column and row (the reference's separable fill caches the same per
    // column, SBInterpolatedImage.cpp:820-866)
    for (int l = 0; l < tpl.n_leaves; ++l) {
        S.ii_cache[l] = -1;
        const LeafParams& L = S.leaf[l];
        if (!II || L.type != GSB_INTERPOLATED || (L.flags & GSB_LEAF_JAC_GENERAL)) continue;
        const int bytes = ((hk + 1 + Nk + 1) * (int)sizeof(IITaps<T>) + 15) & ~15;
        if (used + bytes <= budget) { S.ii_cache[l] = used; used += bytes; }
    }
    for (int p = 0; p < tpl.n_phases; ++p) {
        S.phase_cache[p] = -1;
        if (S.phase_sep[p]) continue;
        const int bytes = ((hk + 1 + Nk + 1) * (int)sizeof(Cx<T>) + 15) & ~15;
        if (used + bytes <= budget) { S.phase_cache[p] = used; used += bytes; }
    }
    for (int l = 0; l < tpl.n_leaves; ++l) {
        const LeafParams& L = S.leaf[l];
        const bool sep = !(L.flags & GSB_LEAF_JAC_GENERAL) && (L.type == GSB_BOX || L.type == GSB_GAUSSIAN);
        if (!sep || S.leaf_sep[l]) continue;
        const int bytes = ((hk + 1 + Nk + 1) * (int)sizeof(T) + 15) & ~15;
        if (used + bytes <= budget) { S.leaf_cache[l] = used; used += bytes; }
    }
}

// Fill the planned caches (whole block).
template <typename T, bool II = true>
__device__ inline void fill_caches(const StampSmem& S, const gsb_template& tpl, unsigned char* cache,
                                   double dk, int Nk)
{
    const int hk = Nk / 2;
    for (int l = 0; l < tpl.n_leaves; ++l) {
        if (II && S.ii_cache[l] >= 0) {
            const LeafParams& L = S.leaf[l];
            IITaps<T>* E = reinterpret_cast<IITaps<T>*>(cache + S.ii_cache[l]);
            for (int t = threadIdx.x; t < hk + 1 + Nk + 1; t += blockDim.x) {
                const bool isx = t <= hk;
                const int idx = isx ? t : t - (hk + 1) - hk;
                // k' as ii_kvalue forms it for a diagonal Jacobian (the zero terms are exact)
                const double kp = isx ? L.jac[0] * (idx * dk) : L.jac[3] * (idx * dk);
                ii_axis_taps<T>(L, kp, true, isx, E[t]);
            }
        }
        if (S.sersic_cache[l] >= 0) {
            typename NodeT<T>::type* dst = reinterpret_cast<typename NodeT<T>::type*>(cache + S.sersic_cache[l]);
            const double4* src = S.sersic[l].node;
            for (int i = threadIdx.x; i < S.sersic[l].n; i += blockDim.x) {
                const double4 v = src[i];
                dst[i].x = T(v.x); dst[i].y = T(v.y); dst[i].z = T(v.z); dst[i].w = T(v.w);
            }
        }
        if (S.leaf_cache[l] >= 0) {
            const LeafParams& L = S.leaf[l];
            T* X = reinterpret_cast<T*>(cache + S.leaf_cache[l]);
            T* Y = X + hk + 1;
            const bool box = L.type == GSB_BOX;
            const double ax = L.jac[0] * dk * (box ? L.d[0] : L.d[0]);
            const double ay = L.jac[3] * dk * (box ? L.d[1] : L.d[0]);
            for (int i = threadIdx.x; i < hk + 1 + Nk + 1; i += blockDim.x) {
                const bool isx = i <= hk;
                const int idx = isx ? i : i - (hk + 1) - hk;
                const T u = T(idx * (isx ? ax : ay));
                const T v = box ? sinc_ref<T>(u) : exp(T(-0.5) * u * u);
                if (isx) X[i] = v; else Y[i - (hk + 1)] = v;
            }
        }
    }
    if (S.xy_cache >= 0) {
        // XS[i] = prod over folded atoms of their kx factor (flux, fs and scales in XS),
        // YS[j + hk] = prod of their ky factor.
        Cx<T>* XS = reinterpret_cast<Cx<T>*>(cache + S.xy_cache);
        Cx<T>* YS = XS + hk + 1;
        for (int t = threadIdx.x; t < hk + 1 + Nk + 1; t += blockDim.x) {
            const bool isx = t <= hk;
            const int idx = isx ? t : t - (hk + 1) - hk;
            Cx<T> v = cx<T>(T(1), T(0));
            for (int l = 0; l < tpl.n_leaves; ++l) {
                if (!S.leaf_sep[l]) continue;
                const LeafParams& L = S.leaf[l];
                const bool box = L.type == GSB_BOX;
                const double ax = L.jac[0] * dk * L.d[0];
                const double ay = L.jac[3] * dk * (box ? L.d[1] : L.d[0]);
                const T u = T(idx * (isx ? ax : ay));
                T f = box ? sinc_ref<T>(u) : exp(T(-0.5) * u * u);
                if (isx) f *= T(L.flux);
                v = cscale<T>(v, f);
            }
            for (int p = 0; p < tpl.n_phases; ++p) {
                if (!S.phase_sep[p]) continue;
                double tt = idx * (isx ? S.phase_ax[p] : S.phase_ay[p]);
                tt -= rint(tt);
                T sn, cs;
                sincospi(T(-2. * tt), &sn, &cs);
                v = cmul<T>(v, cx<T>(cs, sn));
                if (isx) v = cscale<T>(v, T(S.phase[p].flux_scaling));
            }
            if (isx)
                for (int q = 0; q < tpl.n_scales; ++q)
                    if (S.scale_sep[q]) v = cscale<T>(v, T(S.scale[q]));
            if (isx) XS[t] = v; else YS[t - (hk + 1)] = v;
        }
    }
    for (int p = 0; p < tpl.n_phases; ++p) {
        if (S.phase_cache[p] < 0) continue;
        Cx<T>* PX = reinterpret_cast<Cx<T>*>(cache + S.phase_cache[p]);
        Cx<T>* PY = PX + hk + 1;
        for (int i = threadIdx.x; i < hk + 1 + Nk + 1; i += blockDim.x) {
            const bool isx = i <= hk;
            const int idx = isx ? i : i - (hk + 1) - hk;
            double tt = idx * (isx ? S.phase_ax[p] : S.phase_ay[p]);
            tt -= rint(tt);
            T sn, cs;
            sincospi(T(-2. * tt), &sn, &cs);
            if (isx) PX[i] = cx<T>(cs, sn); else PY[i - (hk + 1)] = cx<T>(cs, sn);
        }
    }
}

// Sersic FT from shared-memory nodes (same arithmetic as sersic_kvalue).
template <typename T>
__device__ inline T sersic_kvalue_smem(const SersicTableView& tb, const typename NodeT<T>::type* node, T ksq)
{
    if (ksq >= T(tb.ksq_max)) return (T(tb.highk_a) + T(tb.highk_b) / sqrt(ksq)) / ksq;
    if (ksq < T(tb.ksq_min)) return T(1) + ksq * (T(tb.kderiv2) + ksq * T(tb.kderiv4));
    const T lk = T(0.5) * log(ksq) - T(tb.front);
    const T inv_da = T(1. / tb.da);
    int i = int(ceil(lk * inv_da));
    if (i >= tb.n) i = tb.n - 1;
    if (i <= 0) i = 1;
    const typename NodeT<T>::type n0 = node[i - 1], n1 = node[i];
    // The offset from the upper node is 0.5 ln(k_i^2 / k^2), the log of a ratio near 1, and
    // the spacing is the table's: both accurate in FP32 (a difference of two logs of size ~10,
    // or of rounded node positions, would cost up to ~1e-6 of the value).  bb = h - aa keeps
    // the weights aa / h + bb / h summing to 1.
    const T h = T(tb.da);
    const T aa = T(0.5) * log(n1.w / ksq);
    const T bb = h - aa;
    const T num = aa * n0.y + bb * n1.y - (T(1) / T(6)) * aa * bb * ((aa + h) * n0.z + (bb + h) * n1.z);
    return num / h / ksq;
}

// One leaf at k index (i, j) with the shared-memory caches.
template <typename T>
__device__ __forceinline__ T leaf_fast(const StampSmem& S, const unsigned char* cache, int arg, T kx, T ky,
                                       int i, int j, const GridRef& g)
{
    const int hk = g.n / 2;
    const LeafParams& L = S.leaf[arg];
    if (S.leaf_cache[arg] >= 0) {
        const T* X = reinterpret_cast<const T*>(cache + S.leaf_cache[arg]);
        return T(L.flux) * X[i] * X[hk + 1 + j + hk];
    }
    if (S.sersic_cache[arg] >= 0) {
        const T A = T(L.jac[0]), B = T(L.jac[1]), C = T(L.jac[2]), D = T(L.jac[3]);
        const T kxp = A * kx + C * ky, kyp = B * kx + D * ky;
        const T r0 = T(L.d[0]);
        return T(L.flux) * sersic_kvalue_smem<T>(
                   S.sersic[arg], reinterpret_cast<const typename NodeT<T>::type*>(cache + S.sersic_cache[arg]),
                   (kxp * kxp + kyp * kyp) * r0 * r0);
    }
    return leaf_kvalue<T>(L, S.sersic, kx, ky, g, i - g.x0, j - g.y0);
}

// One leaf as a complex value: InterpolatedImage leaves are complex, the others real.
template <typename T, bool II = true>
__device__ __forceinline__ Cx<T> leaf_cfast(const StampSmem& S, const unsigned char* cache, int arg, T kx, T ky,
                                            int i, int j, const GridRef& g)
{
    if (II && S.leaf[arg].type == GSB_INTERPOLATED) {
        if (S.ii_cache[arg] >= 0) {
            const IITaps<T>* E = reinterpret_cast<const IITaps<T>*>(cache + S.ii_cache[arg]);
            const int hk = g.n / 2;
            return ii_sum<T>(S.leaf[arg], E[i], E[hk + 1 + j + hk]);
        }
        return ii_kvalue<T>(S.leaf[arg], g.dk, i, j);
    }
    return cx<T>(leaf_fast<T>(S, cache, arg, kx, ky, i, j, g), T(0));
}

// Evaluation of the ops [o0, o1) (a complete subtree, or the whole program) with the caches and
// a 4-deep register stack (warp-uniform branches).
template <typename T, bool II = true>
__device__ __forceinline__ Cx<T> eval_range(const gsb_template& tpl, const StampSmem& S,
                                            const unsigned char* cache, double dk, int i, int j,
                                            const GridRef& g, int o0, int o1)
{
    const int hk = g.n / 2;
    Cx<T> s0 = cx<T>(T(0), T(0)), s1 = s0, s2 = s0, s3 = s0;
    int sp = 0;
    const T kx = T(i) * T(dk), ky = T(j) * T(dk);
    for (int o = o0; o < o1; ++o) {
        const int code = tpl.op_code[o], arg = tpl.op_arg[o];
        if (code == GSB_OP_LEAF) {
            const Cx<T> c = leaf_cfast<T, II>(S, cache, arg, kx, ky, i, j, g);
            if (sp == 0) s0 = c; else if (sp == 1) s1 = c; else if (sp == 2) s2 = c; else s3 = c;
            ++sp;
        } else if (code == GSB_OP_MUL || code == GSB_OP_ADD) {
            --sp;
            const bool mul = code == GSB_OP_MUL;
            if (sp == 1) s0 = mul ? cmul<T>(s0, s1) : cadd<T>(s0, s1);
            else if (sp == 2) s1 = mul ? cmul<T>(s1, s2) : cadd<T>(s1, s2);
            else s2 = mul ? cmul<T>(s2, s3) : cadd<T>(s2, s3);
        } else {
            Cx<T> f;
            if (code == GSB_OP_PHASE) {
                const T fs = T(S.phase[arg].flux_scaling);
                if (S.phase_cache[arg] >= 0) {
                    const Cx<T>* PX = reinterpret_cast<const Cx<T>*>(cache + S.phase_cache[arg]);
                    f = cscale<T>(cmul<T>(PX[i], PX[hk + 1 + j + hk]), fs);
                } else {
                    double tt = i * S.phase_ax[arg] + j * S.phase_ay[arg];
                    tt -= rint(tt);
                    T sn, cs;
                    sincospi(T(-2. * tt), &sn, &cs);
                    f = cx<T>(fs * cs, fs * sn);
                }
            } else {
                f = cx<T>(T(S.scale[arg]), T(0));
            }
            if (sp == 1) s0 = cmul<T>(s0, f);
            else if (sp == 2) s1 = cmul<T>(s1, f);
            else if (sp == 3) s2 = cmul<T>(s2, f);
            else s3 = cmul<T>(s3, f);
        }
    }
    return s0;
}

template <typename T, bool II = true>
__device__ __forceinline__ Cx<T> eval_fast(const gsb_template& tpl, const StampSmem& S,
                                           const unsigned char* cache, double dk, int i, int j,
                                           const GridRef& g)
{
    return eval_range<T, II>(tpl, S, cache, dk, i, j, g, 0, tpl.n_ops);
}

// The factored program at (i, j): product of the per-point atoms (real leaves, complex
// subtrees) times the folded separable factors XS[i] YS[j + hk].
template <typename T, bool II = true>
__device__ __forceinline__ Cx<T> eval_factored(const gsb_template& tpl, const StampSmem& S,
                                               const unsigned char* cache, double dk, int i, int j,
                                               const GridRef& g)
{
    const int hk = g.n / 2;
    const T kx = T(i) * T(dk), ky = T(j) * T(dk);
    T r = T(1);
    Cx<T> c = cx<T>(T(1), T(0));
    for (int a = 0; a < S.n_atoms; ++a) {
        const int o0 = S.atom_o0[a], o1 = S.atom_o1[a];
        if (o1 - o0 == 1) {
            const int l = tpl.op_arg[o0];
            if (II && S.leaf[l].type == GSB_INTERPOLATED) c = cmul<T>(c, leaf_cfast<T, II>(S, cache, l, kx, ky, i, j, g));
            else r *= leaf_fast<T>(S, cache, l, kx, ky, i, j, g);
        } else {
            c = cmul<T>(c, eval_range<T, II>(tpl, S, cache, dk, i, j, g, o0, o1));
        }
    }
    const Cx<T>* XS = reinterpret_cast<const Cx<T>*>(cache + S.xy_cache);
    const Cx<T> xy = cmul<T>(XS[i], XS[hk + 1 + j + hk]);
    return cscale<T>(cmul<T>(c, xy), r);
}

// acc += v with Kahan's compensation term comp (componentwise).
template <typename T>
__device__ __forceinline__ void kahan_add(Cx<T>& acc, Cx<T>& comp, Cx<T> v)
{
    const T yx = v.x - comp.x, yy = v.y - comp.y;
    const T tx = acc.x + yx, ty = acc.y + yy;
    comp.x = (tx - acc.x) - yx;
    comp.y = (ty - acc.y) - yy;
    acc.x = tx;
    acc.y = ty;
}

template <typename T>
__device__ inline void store_pixel(void* out, int dtype, int add, long long idx, T v)
{
    if (dtype == GSB_F32) {
        float* o = reinterpret_cast<float*>(out) + idx;
        *o = add ? *o + float(v) : float(v);
    } else {
        double* o = reinterpret_cast<double*>(out) + idx;
        *o = add ? *o + double(v) : double(v);
    }
}

template <typename T, int N>
constexpr size_t smem_bytes(bool wsmem)
{
    size_t off = (sizeof(StampSmem) + 15) & ~size_t(15);
    off += sizeof(Cx<T>) * N * (1 + fused_warps<T, N>());
    if (wsmem) off += sizeof(Cx<T>) * (N / 2 + 1) * (N + 1);
    return ((off + 15) & ~size_t(15)) + kCacheBytes;
}

template <typename T, int N>
constexpr bool w_fits_smem()
{
    return smem_bytes<T, N>(true) <= kSmemLimit;
}

// Resident CTAs per SM that the shared memory allows (at most 2): the register budget is
// capped to match, so that code used only by some programs (the FP64 transform of image
// leaves, the general-Jacobian paths) cannot halve the occupancy of every other program.
constexpr size_t kSmemPerSM = 228 * 1024;

template <typename T, int N>
__host__ __device__ constexpr int fused_min_blocks()
{
    return kSmemPerSM / (smem_bytes<T, N>(w_fits_smem<T, N>()) + 1024) >= 2 ? 2 : 1;
}

template <typename T, int N, bool WSMEM, bool II = true>
__global__ void __launch_bounds__(fused_warps<T, N>() * 32, fused_min_blocks<T, N>()) draw_fused_kernel(const __grid_constant__ DrawArgs a)
{
    constexpr int NW = fused_warps<T, N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int H = N / 2 + 1;
    constexpr int WS = N + 1;   // column stride of W (padding against bank conflicts)
    StampSmem& S = *reinterpret_cast<StampSmem*>(smem_raw);
    size_t off = (sizeof(StampSmem) + 15) & ~size_t(15);
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

    for (int s = blockIdx.x; s < a.n_stamps; s += gridDim.x) {
        __syncthreads();
        load_stamp(S, a.tpl, s, a.leaves, a.phases, a.scales, a.stamps, a.sersic_header,
                   a.sersic_node, a.sersic_stride, 1. / N);
        __syncthreads();
        const int Nk = S.geom.Nk;
        const int hk = Nk / 2;
        const GridRef g{dk, 0, -hk, hk + 1, Nk + 1};
        if (threadIdx.x == 0) plan_caches<T, II>(S, a.tpl, Nk);
        __syncthreads();
        fill_caches<T, II>(S, a.tpl, cache, dk, Nk);
        __syncthreads();
        const bool fast = S.regstack;
        const bool factored = S.xy_cache >= 0;

        // ---- column phase: wrapped k-values, inverse DFT along ky ----
        for (int c = warp; c < H; c += NW) {
            const int alo = ceil_div(-hk - c, N), ahi = floor_div(hk - c, N);
            for (int r = lane; r < N; r += 32) {
                const int kyc = r < N / 2 ? r : r - N;
                const int blo = ceil_div(-hk - kyc, N), bhi = floor_div(hk - kyc, N);
                // the fold (wrap) of the aliases, with Kahan compensation
                Cx<T> acc = cx<T>(T(0), T(0)), comp = acc;
                for (int ia = alo; ia <= ahi; ++ia) {
                    const int kx = c + ia * N;
                    for (int ib = blo; ib <= bhi; ++ib) {
                        const int ky = kyc + ib * N;
                        const bool pos = kx >= 0;
                        const int ii = pos ? kx : -kx, jj = pos ? ky : -ky;
                        Cx<T> v = factored ? eval_factored<T, II>(a.tpl, S, cache, dk, ii, jj, g)
                                  : fast ? eval_fast<T, II>(a.tpl, S, cache, dk, ii, jj, g)
                                         : eval_program<T, II>(a.tpl, S, dk, ii, jj, g);
                        if (!pos) v = cconj<T>(v);
                        kahan_add<T>(acc, comp, v);
                    }
                }
                buf[r] = acc;
            }
            __syncwarp();
            warp_fft<T, N, +1>(buf, tw);
            for (int r = lane; r < N; r += 32) W[(size_t)c * WS + r] = buf[r];
            __syncwarp();
        }
        __syncthreads();

        // ---- row phase: two image rows per complex transform ----
        const gsb_stamp& G = S.geom;
        const int npairs = (G.ny + 1) / 2;
        double fsum = 0., fcomp = 0.;
        for (int p = warp; p < npairs; p += NW) {
            const int py1 = G.ymin + 2 * p;
            const bool two = 2 * p + 1 < G.ny;
            const int y1 = pmod(py1, N), y2 = pmod(py1 + 1, N);
            for (int kx = lane; kx < N; kx += 32) {
                Cx<T> a1, a2;
                if (kx < H) {
                    a1 = W[(size_t)kx * WS + y1];
                    a2 = two ? W[(size_t)kx * WS + y2] : cx<T>(T(0), T(0));
                } else {
                    a1 = cconj<T>(W[(size_t)(N - kx) * WS + y1]);
                    a2 = two ? cconj<T>(W[(size_t)(N - kx) * WS + y2]) : cx<T>(T(0), T(0));
                }
                buf[kx] = cx<T>(a1.x - a2.y, a1.y + a2.x);
            }
            __syncwarp();
            warp_fft<T, N, +1>(buf, tw);
            const long long row1 = G.out_offset + (long long)(2 * p) * G.nx;
            for (int i = lane; i < G.nx; i += 32) {
                const Cx<T> v = buf[pmod(G.xmin + i, N)];
                const T v1 = v.x * inv_n2;
                store_pixel<T>(a.out, a.out_dtype, a.add, row1 + i, v1);
                // Neumaier compensated sum in FP64
                const double x1 = double(v1);
                double tsum = fsum + x1;
                fcomp += fabs(fsum) >= fabs(x1) ? (fsum - tsum) + x1 : (x1 - tsum) + fsum;
                fsum = tsum;
                if (two) {
                    const T v2 = v.y * inv_n2;
                    store_pixel<T>(a.out, a.out_dtype, a.add, row1 + G.nx + i, v2);
                    const double x2 = double(v2);
                    tsum = fsum + x2;
                    fcomp += fabs(fsum) >= fabs(x2) ? (fsum - tsum) + x2 : (x2 - tsum) + fsum;
                    fsum = tsum;
                }
            }
            __syncwarp();
        }
        if (a.added_flux) {
            double v = fsum + fcomp;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) S.flux_part[warp] = v;
            __syncthreads();
            if (threadIdx.x == 0) {
                double tot = 0.;
                for (int w = 0; w < NW; ++w) tot += S.flux_part[w];
                a.added_flux[s] = tot;
            }
        }
    }
}

template <typename T>
__global__ void draw_kimage_kernel(const __grid_constant__ gsb_template tpl, int n_stamps, const gsb_leaf* leaves,
                                   const gsb_phase* phases, const double* scales,
                                   const double* sh, const double4* snode, int sstride, double dk,
                                   int kxmin, int kymin, int nkx, int nky, void* out, int dtype)
{
    __shared__ StampSmem S;
    const long long per = (long long)nkx * nky;
    for (int s = blockIdx.y; s < n_stamps; s += gridDim.y) {
        __syncthreads();
        load_stamp(S, tpl, s, leaves, phases, scales, nullptr, sh, snode, sstride, dk / (2. * kPi));
        __syncthreads();
        const GridRef g{dk, kxmin, kymin, nkx, nky};
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < per;
             p += (long long)gridDim.x * blockDim.x) {
            const int i = int(p % nkx), j = int(p / nkx);
            const Cx<T> v = eval_program<T>(tpl, S, dk, kxmin + i, kymin + j, g);
            const long long o = (s * per + p) * 2;
            if (dtype == GSB_F32) {
                reinterpret_cast<float*>(out)[o] = float(v.x);
                reinterpret_cast<float*>(out)[o + 1] = float(v.y);
            } else {
                reinterpret_cast<double*>(out)[o] = double(v.x);
                reinterpret_cast<double*>(out)[o + 1] = double(v.y);
            }
        }
    }
}

inline bool has_image_leaves(const gsb_template& tpl)
{
    for (int l = 0; l < tpl.n_leaves; ++l)
        if (tpl.leaf_type[l] == GSB_INTERPOLATED) return true;
    return false;
}

template <typename T, int N>
int draw_grid(int n_stamps)
{
    DeviceState* st = device_state();
    const size_t sm = smem_bytes<T, N>(w_fits_smem<T, N>());
    int per_sm = int(std::min<size_t>(kSmemLimit / sm, 4));
    if (per_sm < 1) per_sm = 1;
    return std::max(1, std::min(n_stamps, st->sm_count * per_sm));
}

template <typename T, int N>
size_t workspace_bytes_for(int n_stamps)
{
    if (w_fits_smem<T, N>()) return 0;
    return sizeof(Cx<T>) * (size_t)(N / 2 + 1) * (N + 1) * draw_grid<T, N>(n_stamps);
}

template <typename T, int N>
int launch_fused(const DrawArgs& args, size_t work_bytes, cudaStream_t stream)
{
    constexpr bool wsmem = w_fits_smem<T, N>();
    constexpr size_t sm = smem_bytes<T, N>(wsmem);
    const int grid = draw_grid<T, N>(args.n_stamps);
    if (!wsmem && (args.work == nullptr || work_bytes < workspace_bytes_for<T, N>(args.n_stamps)))
        return set_error(GSB_ERR_INVALID, "draw workspace too small");
    // programs without image leaves run the instance compiled without their code
    if (has_image_leaves(args.tpl)) {
        GSB_CUDA_CHECK(cudaFuncSetAttribute(draw_fused_kernel<T, N, wsmem, true>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        draw_fused_kernel<T, N, wsmem, true><<<grid, fused_warps<T, N>() * 32, sm, stream>>>(args);
    } else {
        GSB_CUDA_CHECK(cudaFuncSetAttribute(draw_fused_kernel<T, N, wsmem, false>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        draw_fused_kernel<T, N, wsmem, false><<<grid, fused_warps<T, N>() * 32, sm, stream>>>(args);
    }
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

}  // namespace gsb
