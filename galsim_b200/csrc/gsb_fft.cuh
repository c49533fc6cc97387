// Per-warp Stockham FFT in shared memory for N = 2^a or 3 * 2^a (N <= 1024).
//
// One warp owns one length-N transform held in a shared-memory buffer.  Each pass of radix
// R (3 first when N has a factor 3, then 4, then a final 2 if needed) reads R inputs per
// butterfly, applies the twiddles, does the R-point DFT in registers and, after a
// __syncwarp, writes the outputs back in Stockham (self-sorting) order, so the result is
// in natural order with no bit reversal.  Twiddles come from a per-block table
// tw[m] = exp(+2 pi i m / N) built in FP64.  SIGN = +1 is the unnormalised inverse DFT
// (FFTW_BACKWARD), SIGN = -1 the forward DFT.
#pragma once

#include <cuda_runtime.h>

namespace gsb {

template <typename T> struct CxT;
template <> struct CxT<float>  { using type = float2; };
template <> struct CxT<double> { using type = double2; };
template <typename T> using Cx = typename CxT<T>::type;

template <typename T> __device__ __forceinline__ Cx<T> cx(T x, T y) { Cx<T> r; r.x = x; r.y = y; return r; }
template <typename T> __device__ __forceinline__ Cx<T> cadd(Cx<T> a, Cx<T> b) { return cx<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ Cx<T> csub(Cx<T> a, Cx<T> b) { return cx<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b)
{ return cx<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename T> __device__ __forceinline__ Cx<T> cconj(Cx<T> a) { return cx<T>(a.x, -a.y); }
template <typename T> __device__ __forceinline__ Cx<T> cscale(Cx<T> a, T s) { return cx<T>(a.x * s, a.y * s); }
// multiply by SIGN * i
template <typename T, int SIGN> __device__ __forceinline__ Cx<T> cmul_si(Cx<T> a)
{ return SIGN > 0 ? cx<T>(-a.y, a.x) : cx<T>(a.y, -a.x); }

template <typename T, int R, int SIGN>
__device__ __forceinline__ void dft_small(Cx<T>* v)
{
    if constexpr (R == 2) {
        const Cx<T> a = v[0], b = v[1];
        v[0] = cadd<T>(a, b);
        v[1] = csub<T>(a, b);
    } else if constexpr (R == 3) {
        const Cx<T> a = v[0], b = v[1], c = v[2];
        const Cx<T> t1 = cadd<T>(b, c);
        const Cx<T> t2 = csub<T>(a, cscale<T>(t1, T(0.5)));
        const Cx<T> t3 = cmul_si<T, SIGN>(cscale<T>(csub<T>(b, c), T(0.86602540378443864676)));
        v[0] = cadd<T>(a, t1);
        v[1] = cadd<T>(t2, t3);
        v[2] = csub<T>(t2, t3);
    } else if constexpr (R == 4) {
        const Cx<T> a = v[0], b = v[1], c = v[2], d = v[3];
        const Cx<T> s0 = cadd<T>(a, c), s1 = csub<T>(a, c);
        const Cx<T> s2 = cadd<T>(b, d), s3 = cmul_si<T, SIGN>(csub<T>(b, d));
        v[0] = cadd<T>(s0, s2);
        v[1] = cadd<T>(s1, s3);
        v[2] = csub<T>(s0, s2);
        v[3] = csub<T>(s1, s3);
    }
}

template <typename T, int N, int R, int NS, int SIGN>
__device__ __forceinline__ void stockham_pass(Cx<T>* buf, const Cx<T>* tw, int lane)
{
    constexpr int NB = N / R;
    constexpr int PER = (NB + 31) / 32;
    constexpr int TSTEP = N / (NS * R);
    Cx<T> v[PER][R];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int b = lane + 32 * t;
        if (NB % 32 == 0 || b < NB) {
            const int k = b % NS;
#pragma unroll
            for (int r = 0; r < R; ++r) v[t][r] = buf[b + r * NB];
#pragma unroll
            for (int r = 1; r < R; ++r) {
                // r k TSTEP <= (R - 1)(NS - 1) N / (NS R) < N: no reduction mod N needed
                const int idx = r * k * TSTEP;
                Cx<T> w = tw[idx];
                if (SIGN < 0) w.y = -w.y;
                v[t][r] = cmul<T>(v[t][r], w);
            }
            dft_small<T, R, SIGN>(v[t]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < PER; ++t) {
        const int b = lane + 32 * t;
        if (NB % 32 == 0 || b < NB) {
            const int k = b % NS;
            const int base = (b / NS) * NS * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[base + r * NS] = v[t][r];
        }
    }
    __syncwarp();
}

template <typename T, int N, int NS, int SIGN>
__device__ __forceinline__ void fft_passes(Cx<T>* buf, const Cx<T>* tw, int lane)
{
    if constexpr (NS < N) {
        constexpr int rem = N / NS;
        constexpr int R = (NS == 1 && (N % 3) == 0) ? 3 : ((rem % 4) == 0 ? 4 : 2);
        stockham_pass<T, N, R, NS, SIGN>(buf, tw, lane);
        fft_passes<T, N, NS * R, SIGN>(buf, tw, lane);
    }
}

// In-place length-N DFT of buf (shared memory) by the calling warp.  All 32 lanes must call.
template <typename T, int N, int SIGN>
__device__ __forceinline__ void warp_fft(Cx<T>* buf, const Cx<T>* tw)
{
    fft_passes<T, N, 1, SIGN>(buf, tw, threadIdx.x & 31);
}

// tw[m] = exp(+2 pi i m / N), filled by the whole block.
template <typename T>
__device__ inline void fill_twiddles(Cx<T>* tw, int N)
{
    for (int m = threadIdx.x; m < N; m += blockDim.x) {
        double s, c;
        sincospi(2.0 * m / N, &s, &c);
        tw[m] = cx<T>(T(c), T(s));
    }
}

constexpr int kBlockFftMaxPerThread = 4;   // N / R <= 4096 butterflies per pass at 1024 threads

// Block-wide in-place Stockham FFT of length N (2^a or 3 * 2^a, N / R <= blockDim.x *
// kBlockFftMaxPerThread) in shared memory, the same radix plan as warp_fft; all threads of the
// block must call.  tw: exp(+2 pi i m / N) for m < N (global, FP64).
template <typename T, int SIGN>
__device__ void block_fft(Cx<T>* buf, int N, const double2* __restrict__ tw)
{
    int NS = 1;
    while (NS < N) {
        const int rem = N / NS;
        const int R = (NS == 1 && N % 3 == 0) ? 3 : ((rem % 4) == 0 ? 4 : 2);
        const int NB = N / R;
        const int tstep = N / (NS * R);
        Cx<T> v[kBlockFftMaxPerThread][4];
#pragma unroll
        for (int t = 0; t < kBlockFftMaxPerThread; ++t) {
            const int b = threadIdx.x + t * blockDim.x;
            if (b < NB) {
                const int k = b % NS;
                for (int r = 0; r < R; ++r) v[t][r] = buf[b + r * NB];
                for (int r = 1; r < R; ++r) {
                    // r k tstep <= (R - 1)(NS - 1) N / (NS R) < N
                    const double2 w = __ldg(&tw[r * k * tstep]);
                    v[t][r] = cmul<T>(v[t][r], cx<T>(T(w.x), SIGN > 0 ? T(w.y) : T(-w.y)));
                }
                if (R == 4) dft_small<T, 4, SIGN>(v[t]);
                else if (R == 3) dft_small<T, 3, SIGN>(v[t]);
                else dft_small<T, 2, SIGN>(v[t]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < kBlockFftMaxPerThread; ++t) {
            const int b = threadIdx.x + t * blockDim.x;
            if (b < NB) {
                const int k = b % NS;
                const int base = (b / NS) * NS * R + k;
                for (int r = 0; r < R; ++r) buf[base + r * NS] = v[t][r];
            }
        }
        __syncthreads();
        NS *= R;
    }
}

}  // namespace gsb
