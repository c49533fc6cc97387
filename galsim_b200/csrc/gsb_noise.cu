// Noise on device stamps: GaussianNoise, PoissonNoise and CCDNoise with the reference's random
// streams.
//
// Reference: galsim/noise.py (GaussianNoise._applyTo :259-263, PoissonNoise._applyTo :331-356,
// CCDNoise._applyTo :463-486), src/Random.cpp (BaseDeviate::seed :156-191, generate /
// addGenerate :204-270, PoissonDeviate :498-606) and the Boost.Random 1.48 engines and
// distributions it uses:
//   * mt19937, seeded with the third draw of an mt11213b seeded with the user's seed (the
//     Mersenne Twister of Matsumoto & Nishimura 1998 with the 2002 init_genrand seeding);
//   * uniform_01 on a 32-bit engine: one draw times 2^-32;
//   * normal_distribution: Box-Muller pairs, rho = sqrt(-2 ln(1 - u2)), cos(2 pi u1) first,
//     then sin (the pair is cached between calls, cleared by clearCache);
//   * poisson_distribution: inversion below mean 10, otherwise the PTRD transformed rejection
//     of W. Hoermann (Insurance: Mathematics and Economics 12, 1993), one or more draws each;
//     PoissonDeviate switches to a normal with sigma = sqrt(mean) above 2^30.
//
// One warp per stamp holds the 624-word state in shared memory and regenerates it
// cooperatively (the twist in 32-word chunks, whose dependences span 227 and 397 words).
// Gaussian pairs are independent once their two words are known, so the lanes take consecutive
// pairs of each block.  Poisson draws consume a data-dependent number of words; the warp draws
// 32 pixels at a time speculatively and keeps the prefix whose stream positions were right
// (pass 2, between a parallel pass for the expectations and a pass for the read noise and the
// cast).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gsb_internal.cuh"

namespace gsb {
namespace {

constexpr int kMtN = 624, kMtM = 397;
constexpr uint32_t kMtA = 0x9908b0dfu;
constexpr int kNoiseWarps = 8;

__device__ __forceinline__ uint32_t mt_temper(uint32_t z)
{
    z ^= z >> 11;
    z ^= (z << 7) & 0x9d2c5680u;
    z ^= (z << 15) & 0xefc60000u;
    z ^= z >> 18;
    return z;
}

__device__ __forceinline__ uint32_t mt_mix(uint32_t xj, uint32_t xj1, uint32_t xm)
{
    const uint32_t y = (xj & 0x80000000u) | (xj1 & 0x7fffffffu);
    return xm ^ (y >> 1) ^ ((xj1 & 1u) * kMtA);
}

// In-place twist of the mt19937 state by the calling warp.
__device__ void mt_twist(uint32_t* x, int lane)
{
    // x[j] for j < n - m reads x[j + m] (old); later j read x[j - (n - m)] (already new); the
    // distance 227 exceeds a chunk, so chunks of 32 in order see exactly the sequential values.
    for (int j0 = 0; j0 < kMtN - 1; j0 += 32) {
        const int j = j0 + lane;
        uint32_t v = 0;
        if (j < kMtN - 1) {
            const uint32_t xm = j < kMtN - kMtM ? x[j + kMtM] : x[j - (kMtN - kMtM)];
            v = mt_mix(x[j], x[j + 1], xm);
        }
        __syncwarp();
        if (j < kMtN - 1) x[j] = v;
        __syncwarp();
    }
    if (lane == 0) x[kMtN - 1] = mt_mix(x[kMtN - 1], x[0], x[kMtM - 1]);
    __syncwarp();
}

// BaseDeviate(seed): mt11213b(seed), two draws discarded, the third seeds the mt19937; the
// state is left at the end of its block, so the first draw twists.  Sequential, one thread.
__device__ void mt_seed_body(uint32_t* x, long long seed)
{
    // mt11213b: w 32, n 351, m 175, r 19, a 0xccab8ee7, tempering (11, 7 0x31b6ab00,
    // 15 0xffe50000, 17); the first 351 words of the buffer serve as its state
    constexpr int n = 351, m = 175;
    uint32_t* a = x;
    a[0] = uint32_t(seed);
    for (int i = 1; i < n; ++i) a[i] = 1812433253u * (a[i - 1] ^ (a[i - 1] >> 30)) + uint32_t(i);
    uint32_t out = 0;
    for (int k = 0; k < 3; ++k) {    // draws 0 and 1 are discarded
        // only the first three words of the twisted state are needed: x'[k] = x[k+m] ^ mix(x[k], x[k+1])
        const uint32_t y = (a[k] & 0xfff80000u) | (a[k + 1] & 0x0007ffffu);
        uint32_t z = a[k + m] ^ (y >> 1) ^ ((a[k + 1] & 1u) * 0xccab8ee7u);
        z ^= z >> 11;
        z ^= (z << 7) & 0x31b6ab00u;
        z ^= (z << 15) & 0xffe50000u;
        z ^= z >> 17;
        out = z;
    }
    x[0] = out;
    for (int i = 1; i < kMtN; ++i) x[i] = 1812433253u * (x[i - 1] ^ (x[i - 1] >> 30)) + uint32_t(i);
    if ((x[0] & 0x80000000u) == 0) {
        bool zero = true;
        for (int i = 1; i < kMtN && zero; ++i) zero = x[i] == 0;
        if (zero) x[0] = 0x80000000u;
    }
}

__device__ void mt_seed(uint32_t* x, long long seed, int lane)
{
    if (lane == 0) mt_seed_body(x, seed);
    __syncwarp();
}

// A warp's position in its stream: the state x (shared), the index i of the next word in the
// current block (kMtN = exhausted), and the count of words consumed since seeding.  The words
// themselves are read block by block (gaussian_run); skip moves the position.
struct WarpStream {
    uint32_t* x;
    int i;
    long long used;
    int lane;

    __device__ void skip(long long n)
    {
        while (n > 0) {
            if (i == kMtN) { mt_twist(x, lane); i = 0; }
            const long long take = n < (long long)(kMtN - i) ? n : (long long)(kMtN - i);
            i += int(take);
            used += take;
            n -= take;
        }
    }
};

constexpr double kPi2 = 2. * 3.14159265358979323846;

// Box-Muller pair from its two words: deviate 0 = rho cos(2 pi u1), deviate 1 = rho sin.
__device__ __forceinline__ void bm_pair(uint32_t w1, uint32_t w2, double& c, double& s)
{
    const double r1 = double(w1) * (1. / 4294967296.);
    const double r2 = double(w2) * (1. / 4294967296.);
    const double rho = sqrt(-2. * log(1. - r2));
    c = rho * cos(kPi2 * r1);
    s = rho * sin(kPi2 * r1);
}

template <typename T>
__device__ __forceinline__ T* pix_ptr(void* img, long long off) { return reinterpret_cast<T*>(img) + off; }

// Gaussian deviates d_j = sigma * N_j for j = 0..n-1 from a fresh pair cache at the stream's
// position: pair m uses the words at positions 2m and 2m + 1 from here.  op(j, d) consumes them.
template <typename Op>
__device__ void gaussian_run(WarpStream& st, long long n, double sigma, Op op)
{
    const int lane = st.lane;
    const long long npairs = (n + 1) / 2;
    long long m0 = 0;                   // first pair not yet produced
    while (m0 < npairs) {
        if (st.i == kMtN) {
            mt_twist(st.x, lane);
            st.i = 0;
        }
        // pairs whose second word lies in this block, starting at the current index i
        // (word of pair m0 + k: first at i + 2k, second at i + 2k + 1)
        const int avail = kMtN - st.i;                 // words left in the block
        const long long np = min((long long)(avail / 2), npairs - m0);
        for (long long k = lane; k < np; k += 32) {
            const int p = st.i + int(2 * k);
            double c, s;
            bm_pair(mt_temper(st.x[p]), mt_temper(st.x[p + 1]), c, s);
            const long long j = 2 * (m0 + k);
            op(j, c * sigma);
            if (j + 1 < n) op(j + 1, s * sigma);
        }
        m0 += np;
        st.i += int(2 * np);
        st.used += 2 * np;
        if (m0 < npairs && st.i == kMtN - 1) {
            // a pair straddling two blocks: its first word ends this block
            const uint32_t w1 = mt_temper(st.x[kMtN - 1]);
            mt_twist(st.x, lane);
            const uint32_t w2 = mt_temper(st.x[0]);
            st.i = 1;
            st.used += 2;
            if (lane == 0) {
                double c, s;
                bm_pair(w1, w2, c, s);
                const long long j = 2 * m0;
                op(j, c * sigma);
                if (j + 1 < n) op(j + 1, s * sigma);
            }
            ++m0;
        }
    }
    __syncwarp();
}

// Uniform deviates u_j = word_j 2^-32 (boost uniform_01 on the 32-bit engine: one word each)
// for j = 0..n-1 from the stream's position; op(j, u) consumes them.
template <typename Op>
__device__ void uniform_run(WarpStream& st, long long n, Op op)
{
    long long m0 = 0;
    while (m0 < n) {
        if (st.i == kMtN) {
            mt_twist(st.x, st.lane);
            st.i = 0;
        }
        const long long take = min((long long)(kMtN - st.i), n - m0);
        for (long long k = st.lane; k < take; k += 32)
            op(m0 + k, double(mt_temper(st.x[st.i + int(k)])) * (1. / 4294967296.));
        m0 += take;
        st.i += int(take);
        st.used += take;
        __syncwarp();
    }
}

// log k! for k < 10 (the table PTRD uses below the Stirling branch).
__device__ __forceinline__ double log_factorial_small(int k)
{
    double r = 0.;
    for (int i = 2; i <= k; ++i) r += log(double(i));
    return r;
}

// The constants of Hoermann's PTRD for one mean (Boost's poisson_distribution, mean >= 10)
// that the speculative pass needs before the draw: sqrt(mean), b and v_r (a and 1/alpha follow
// from b in the draw).
struct PtrdSetup {
    double smu, b, v_r;
};

__device__ __forceinline__ PtrdSetup ptrd_setup(double mean)
{
    PtrdSetup c;
    c.smu = sqrt(mean);
    c.b = 0.931 + 2.53 * c.smu;
    c.v_r = 0.9277 - 3.6224 / (c.b - 2);
    return c;
}

template <typename Stream>
__device__ double ptrd_draw(Stream& st, double mean, const PtrdSetup& c);

// One Poisson draw from the stream.
template <typename Stream>
__device__ double poisson_draw(Stream& st, double mean)
{
    if (mean < 10.) {
        double p = exp(-mean);
        double x = 0.;
        double u = st.uniform();
        // ends once the cumulative probability reaches u <= 1 - 2^-32 (x well below 100 for
        // mean < 10); the bound only guards against a non-finite mean
        while (u > p && x < 1000. && st.ok()) {
            u = u - p;
            x += 1.;
            p = mean * p / x;
        }
        return x;
    }
    return ptrd_draw(st, mean, ptrd_setup(mean));
}

// One attempt of the PTRD loop whose first uniform v missed the immediate region
// (v > 0.86 v_r); w is the attempt's second uniform (the loop reads exactly one more word in
// either branch).  Returns true, with *k the deviate, when the attempt is accepted; a rejected
// attempt leaves nothing behind, the next one starts afresh at the following word.
__device__ __forceinline__ bool ptrd_attempt2(double v, double w, double mean, const PtrdSetup& c, double a,
                                              double inv_alpha, double* k_out)
{
    double u;
    if (v >= c.v_r) {
        u = w - 0.5;
    } else {
        u = v / c.v_r - 0.93;
        u = ((u < 0) ? -0.5 : 0.5) - u;
        v = w * c.v_r;
    }
    const double us = 0.5 - fabs(u);
    if (us < 0.013 && v > us) return false;
    const double k = floor((2 * a / us + c.b) * u + mean + 0.445);
    v = v * inv_alpha / (a / (us * us) + c.b);
    const double log_sqrt_2pi = 0.91893853320467267;
    *k_out = k;
    if (k >= 10) {
        return log(v * c.smu) <= (k + 0.5) * log(mean / k) - mean - log_sqrt_2pi + k -
                                     (1 / 12. - (1 / 360. - 1 / (1260. * k * k)) / (k * k)) / k;
    }
    if (k >= 0) return log(v) <= k * log(mean) - mean - log_factorial_small(int(k));
    return false;
}

__device__ __forceinline__ double ptrd_a(const PtrdSetup& c) { return -0.059 + 0.02483 * c.b; }
__device__ __forceinline__ double ptrd_inv_alpha(const PtrdSetup& c) { return 1.1239 + 1.1328 / (c.b - 3.4); }

// At most this many PTRD attempts per deviate (the rejection loop accepts with probability
// > 0.8 per attempt, so the bound is never reached; it keeps every loop finite).
constexpr int kPtrdMaxAttempts = 1 << 20;

// The PTRD draw (mean >= 10) with its constants already formed.
template <typename Stream>
__device__ double ptrd_draw(Stream& st, double mean, const PtrdSetup& c)
{
    const double a = ptrd_a(c), inv_alpha = ptrd_inv_alpha(c);
    for (int iter = 0; iter < kPtrdMaxAttempts; ++iter) {
        if (!st.ok()) return 0.;
        const double v = st.uniform();
        if (v <= 0.86 * c.v_r) {
            const double u = v / c.v_r - 0.43;
            return floor((2 * a / (0.5 - fabs(u)) + c.b) * u + mean + 0.445);
        }
        const double w = st.uniform();
        double k;
        if (ptrd_attempt2(v, w, mean, c, a, inv_alpha, &k)) return k;
    }
    return mean;   // unreachable in practice (see kPtrdMaxAttempts)
}

struct NoiseArgs {
    int kind;
    gsb_noise_params p;
    const gsb_noise_stamp* stamps;
    int n_stamps;
    void* image;
    int dtype;
    double* scratch;       // FP64 value per pixel (Poisson / CCD; the variances of variable
                           // Gaussian noise), indexed like the image
    long long* used;       // draws used per stamp (Poisson pass -> read-noise pass)
};

// A double as a pixel of type T the way the reference's numpy casts it (astype / copyto with
// casting='unsafe', a C conversion on x86): floats round to nearest; integers truncate toward
// zero and keep the low bits of the type's width (a negative value in an unsigned image wraps,
// as x86's conversion through a wider signed integer leaves it).
template <typename T>
__device__ __forceinline__ T to_pixel(double v) { return T(v); }
template <>
__device__ __forceinline__ int16_t to_pixel<int16_t>(double v) { return int16_t(int(v)); }
template <>
__device__ __forceinline__ uint16_t to_pixel<uint16_t>(double v) { return uint16_t(int(v)); }
template <>
__device__ __forceinline__ int32_t to_pixel<int32_t>(double v) { return int32_t(v); }
template <>
__device__ __forceinline__ uint32_t to_pixel<uint32_t>(double v) { return uint32_t((long long)v); }

// pixel += noise.astype(T): in the pixel type, integers wrapping at their width
template <typename T>
__device__ __forceinline__ T add_pixel(T a, double d) { return a + to_pixel<T>(d); }
template <>
__device__ __forceinline__ int32_t add_pixel<int32_t>(int32_t a, double d)
{
    return int32_t(uint32_t(a) + uint32_t(to_pixel<int32_t>(d)));
}
template <>
__device__ __forceinline__ int16_t add_pixel<int16_t>(int16_t a, double d) { return int16_t(a + to_pixel<int16_t>(d)); }
template <>
__device__ __forceinline__ uint16_t add_pixel<uint16_t>(uint16_t a, double d) { return uint16_t(a + to_pixel<uint16_t>(d)); }

// The cast back into the image and the sky bookkeeping of PoissonNoise / CCDNoise._applyTo:
// frac_sky is subtracted in FP64 before the cast, int_sky after it (in the image type when the
// caller's int_sky has the image's type, as Image.__isub__ does).
template <typename T>
__device__ __forceinline__ T finish_pixel(double w, const gsb_noise_params& p)
{
    if (p.frac_sky != 0.) w -= p.frac_sky;
    T out = to_pixel<T>(w);
    if (p.int_sky != 0.)
        out = p.int_sky_same_dtype ? T(out - T(p.int_sky)) : to_pixel<T>(double(out) - p.int_sky);
    return out;
}

// GaussianNoise: one warp per stamp, the deviates added to the pixels in the image type.
template <typename T>
__global__ void __launch_bounds__(kNoiseWarps * 32) gauss_kernel(const __grid_constant__ NoiseArgs a)
{
    __shared__ uint32_t state[kNoiseWarps][kMtN];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kNoiseWarps + warp;
    if (s >= a.n_stamps) return;
    const gsb_noise_stamp sp = a.stamps[s];
    WarpStream st{state[warp], kMtN, 0, lane};
    mt_seed(st.x, sp.seed, lane);
    st.skip(sp.skip);
    T* img = pix_ptr<T>(a.image, sp.offset);
    if (a.kind == GSB_NOISE_UNIFORM) {
        uniform_run(st, sp.npix, [&](long long j, double u) { img[j] = add_pixel<T>(img[j], u); });
    } else if (a.kind == GSB_NOISE_VARIABLE_GAUSSIAN) {
        // unit deviates scaled by each pixel's own sigma (GaussianDeviate::generateFromVariance)
        const double* var = a.scratch + sp.offset;
        gaussian_run(st, sp.npix, 1., [&](long long j, double d) { img[j] = add_pixel<T>(img[j], d * sqrt(var[j])); });
    } else {
        gaussian_run(st, sp.npix, a.p.sigma, [&](long long j, double d) { img[j] = add_pixel<T>(img[j], d); });
    }
    if (lane == 0 && a.used) a.used[s] = st.used;      // draws consumed since seeding
}

// Poisson / CCD pass 1: the expectation of every pixel (image + sky, in electrons, clipped).
// grid = (chunks, stamps).
template <typename T>
__global__ void expect_kernel(const __grid_constant__ NoiseArgs a)
{
    const gsb_noise_stamp sp = a.stamps[blockIdx.y];
    const T* img = pix_ptr<T>(a.image, sp.offset);
    double* w = a.scratch + sp.offset;
    const bool ccd = a.kind == GSB_NOISE_CCD;
    const double gain = ccd ? a.p.gain : 1.;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < sp.npix;
         j += (long long)gridDim.x * blockDim.x) {
        double v = double(img[j]);
        if (a.p.sky_level != 0.) v += a.p.sky_level;
        if (!ccd || gain > 0.) {
            if (ccd) v *= gain;
            if (v < 0.) v = 0.;
        }
        w[j] = v;
    }
}

// Poisson / CCD pass 2: the draws in pixel order, as PoissonDeviate generateFromExpectation
// (with its mean switching and the normal branch above 2^30, whose pair cache persists while
// the mean is unchanged).  The stream is sequential -- a draw takes a data-dependent number of
// words -- but most draws take exactly one (inversion always; PTRD when its first uniform
// lands in the immediate-acceptance region), so the warp speculates: each lane draws one pixel
// of the next 32 from the position it would have if every earlier nonzero pixel took one word,
// and the pixels up to and including the first one that took a different count are committed
// (their starting positions were right).  Words come from a shared window of two 624-word
// blocks; a draw that would run past it, and the normal branch, are done by the whole warp in
// order.  The result is the sequential stream exactly.
struct Window {
    uint32_t* x;        // mt19937 state of the last generated block
    uint32_t* win;      // tempered words of blocks [wstart / 624, wstart / 624 + 2)
    long long wstart;
    int lane;

    __device__ void gen(uint32_t* dst)
    {
        mt_twist(x, lane);
        for (int j = lane; j < kMtN; j += 32) dst[j] = mt_temper(x[j]);
        __syncwarp();
    }
    __device__ void advance()
    {
        for (int j = lane; j < kMtN; j += 32) win[j] = win[kMtN + j];
        __syncwarp();
        gen(win + kMtN);
        wstart += kMtN;
    }
};

// The whole warp reading in order, advancing the window as needed (collective).
struct WindowStream {
    Window* w;
    long long pos;
    __device__ double uniform()
    {
        while (pos >= w->wstart + 2 * kMtN) w->advance();
        const uint32_t v = w->win[pos - w->wstart];
        ++pos;
        return double(v) * (1. / 4294967296.);
    }
    __device__ bool ok() const { return true; }
};

// Exclusive prefix sum over the warp of per-lane word counts in {0, 1, 2}, and their total:
// two ballots and population counts instead of a chain of shuffles.
struct WarpCounts {
    int excl, total;
};

__device__ __forceinline__ WarpCounts warp_counts012(int g, int lane)
{
    const unsigned lt = (1u << lane) - 1u;
    const unsigned b1 = __ballot_sync(0xffffffffu, g >= 1);
    const unsigned b2 = __ballot_sync(0xffffffffu, g >= 2);
    return WarpCounts{__popc(b1 & lt) + __popc(b2 & lt), __popc(b1) + __popc(b2)};
}

constexpr int kPoissonWarps = 4;      // 7.3 KB of state and window per warp
// Rounds of the fixed point of assumed word counts; each round extends the settled prefix past
// one more two-word pixel, and the commit is bounded by the first rejected attempt anyway.
constexpr int kFixedPointRounds = 4;

__global__ void __launch_bounds__(kPoissonWarps * 32) poisson_kernel(const __grid_constant__ NoiseArgs a)
{
    __shared__ uint32_t state[kPoissonWarps][kMtN];
    __shared__ uint32_t window[kPoissonWarps][2 * kMtN];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kPoissonWarps + warp;
    if (s >= a.n_stamps) return;
    const gsb_noise_stamp sp = a.stamps[s];
    const bool ccd = a.kind == GSB_NOISE_CCD;
    const double gain = ccd ? a.p.gain : 1.;
    if (ccd && !(gain > 0.)) {
        if (lane == 0) a.used[s] = sp.skip;
        return;
    }
    mt_seed(state[warp], sp.seed, lane);
    Window W{state[warp], window[warp], 0, lane};
    const long long skip_blocks = sp.skip / kMtN;
    for (long long b = 0; b < skip_blocks; ++b) mt_twist(W.x, lane);
    W.wstart = skip_blocks * kMtN;
    W.gen(W.win);
    W.gen(W.win + kMtN);
    double* w = a.scratch + sp.offset;
    const long long n = sp.npix;
    const double kMaxPoisson = double(1 << 30);
    long long p0 = 0, base = sp.skip;
    // normal-branch state (PoissonDeviate above 2^30)
    double cur_mean = 1.;
    bool gd_exists = false, gd_valid = false;
    double gd_rho = 0., gd_r1 = 0.;
    // the means of this chunk (p0 + lane) and of the next (p0 + 32 + lane): the next chunk is
    // loaded a round ahead, so the load is off the chain of dependent rounds
    int rejected = 0;          // rejected PTRD attempts on the unfinished pixel at p0
    double m_cur = lane < n ? w[lane] : 0.;
    double m_nxt = 32 + lane < n ? w[32 + lane] : 0.;
    while (p0 < n) {
        while (base >= W.wstart + kMtN) W.advance();
        const long long p_start = p0;
        const long long j = p0 + lane;
        const bool valid = j < n;
        const double mean = valid ? m_cur : 0.;
        const bool nz = valid && mean > 0.;
        const bool special = nz && mean > kMaxPoisson;
        // Assumed word counts: 1 for a draw whose first word lands in the immediate region
        // (inversion always), 2 for the others (their common case), 0 for zero means.  The
        // positions follow from the counts and the counts from the words at the positions, so
        // a few rounds find the consistent assignment (the prefix that matters converges first).
        int guess = nz ? 1 : 0;
        int offs = 0;
        double v0 = 0.;
        PtrdSetup cs{0., 0., 0.};
        if (nz && !special && !(mean < 10.)) cs = ptrd_setup(mean);
        const double v_r = cs.v_r;
        // the immediate region as a bound on the raw word: word * 2^-32 <= 0.86 v_r exactly when
        // word <= floor(0.86 v_r 2^32) (0.4 < v_r < 1 for mean >= 10); every word for inversion
        const uint32_t imm_max = (mean < 10. || special) ? 0xffffffffu
                                                          : uint32_t(floor(0.86 * v_r * 4294967296.));
        for (int round = 0; round < kFixedPointRounds; ++round) {
            offs = warp_counts012(guess, lane).excl;
            const int g2 = nz ? (W.win[int(base - W.wstart) + offs] <= imm_max ? 1 : 2) : 0;
            const bool same = __all_sync(0xffffffffu, g2 == guess);
            guess = g2;
            if (same) break;
        }
        const WarpCounts wc = warp_counts012(guess, lane);
        offs = wc.excl;
        // every lane's draw at its assumed position (all in parallel): one PTRD attempt per lane;
        // a rejected attempt (its two words consumed) leaves its pixel unfinished, to start
        // afresh at the next word in the next round
        double value = mean;
        int count = 0;
        bool bad = special;
        bool unfinished = false;
        if (nz && !special) {
            const int wpos = int(base - W.wstart) + offs;
            v0 = double(W.win[wpos]) * (1. / 4294967296.);
            if (mean < 10.) {
                double pp = exp(-mean), x = 0., u = v0;
                while (u > pp && x < 1000.) {
                    u = u - pp;
                    x += 1.;
                    pp = mean * pp / x;
                }
                value = x;
                count = 1;
            } else {
                // mean >= 10: the immediate formula and the two-word attempt are both evaluated
                // (straight-line, so their latencies overlap instead of running as two divergent
                // paths); the lane keeps the one its first word selects
                const double a_ = ptrd_a(cs);
                const double u = v0 / v_r - 0.43;
                const double val_imm = floor((2 * a_ / (0.5 - fabs(u)) + cs.b) * u + mean + 0.445);
                const bool in_window = wpos + 1 < 2 * kMtN;
                const double w2 = double(W.win[in_window ? wpos + 1 : wpos]) * (1. / 4294967296.);
                double k = 0.;
                const bool accepted = ptrd_attempt2(v0, w2, mean, cs, a_, ptrd_inv_alpha(cs), &k);
                if (v0 <= 0.86 * v_r) {
                    value = val_imm;
                    count = 1;
                } else if (in_window) {
                    unfinished = !accepted;
                    value = k;
                    count = 2;
                } else {
                    bad = true;        // the attempt's second word is past the window
                }
            }
        }
        // the prefix whose positions are right: up to the first lane whose count differs from
        // its assumption or whose pixel is unfinished (that lane's own start is right, so its
        // draw is kept when finished, its consumed words when not, unless it must be redone in
        // order: the normal branch, or a draw past the window)
        const bool fail = valid && (bad || count != guess || unfinished);
        const unsigned fmask = __ballot_sync(0xffffffffu, fail);
        const int nvalid = int(min((long long)32, n - p0));
        const int f = fmask ? __ffs(fmask) - 1 : nvalid;
        const int f_state = fmask ? __shfl_sync(0xffffffffu, bad ? 2 : (unfinished ? 1 : 0), f) : 0;
        const bool f_bad = f_state == 2, f_unf = f_state == 1;
        const int ncommit = f + ((fmask && f_state == 0) ? 1 : 0);
        const bool commit = lane < ncommit && valid;
        if (commit && nz) w[j] = ccd ? value / gain : value;
        // the committed lanes before f used exactly their assumed counts (offs at f); f itself,
        // when committed, its real count
        long long used_words = fmask ? __shfl_sync(0xffffffffu, f_bad ? offs : offs + count, f) : wc.total;
        // a committed ordinary draw replaces the normal branch's deviate (its pair cache goes)
        const unsigned pdmask = __ballot_sync(0xffffffffu, commit && nz);
        if (pdmask) {
            const int last = 31 - __clz(pdmask);
            cur_mean = __shfl_sync(0xffffffffu, mean, last);
            gd_exists = false;
            gd_valid = false;
        }
        base += used_words;
        p0 += ncommit;
        __syncwarp();
        if (f_unf) {
            // rejected attempts on the pixel now at p0 (the PTRD loop's bound, never reached)
            rejected = (ncommit == 0) ? rejected + 1 : 1;
            if (rejected >= kPtrdMaxAttempts) {
                if (lane == 0) w[p0] = ccd ? w[p0] / gain : w[p0];
                __syncwarp();
                ++p0;
                rejected = 0;
            }
        } else {
            rejected = 0;
        }
        if (fmask && f_bad) {
            // the pixel at p0 in order by the whole warp: the normal branch, or a draw that ran
            // past the window
            const double m = w[p0];
            WindowStream ws{&W, base};
            double v;
            if (m > kMaxPoisson) {
                if (m != cur_mean) {
                    cur_mean = m;
                    if (!gd_exists) { gd_exists = true; gd_valid = false; }
                }
                const double sg = sqrt(m);
                if (!gd_valid) {
                    gd_r1 = ws.uniform();
                    const double r2 = ws.uniform();
                    gd_rho = sqrt(-2. * log(1. - r2));
                    gd_valid = true;
                    v = gd_rho * cos(kPi2 * gd_r1) * sg + m;
                } else {
                    gd_valid = false;
                    v = gd_rho * sin(kPi2 * gd_r1) * sg + m;
                }
            } else {
                v = poisson_draw(ws, m);
                cur_mean = m;
                gd_exists = false;
                gd_valid = false;
            }
            __syncwarp();
            if (lane == 0) w[p0] = ccd ? v / gain : v;
            __syncwarp();
            base = ws.pos;
            ++p0;
        }
        // advance the two chunks of means by the d pixels this round finished (0 <= d <= 32:
        // at most 32 commits, or at most 31 and one pixel in order; 0 when the first pixel's
        // attempt was rejected)
        const int src = lane + int(p0 - p_start);
        const double from_cur = __shfl_sync(0xffffffffu, m_cur, src & 31);
        const double from_nxt = __shfl_sync(0xffffffffu, m_nxt, src & 31);
        m_cur = p0 + lane < n ? (src < 32 ? from_cur : from_nxt) : 0.;
        m_nxt = p0 + 32 + lane < n ? w[p0 + 32 + lane] : 0.;
    }
    if (lane == 0) a.used[s] = base;
}

// Poisson / CCD pass 3: the CCD read noise (a fresh Gaussian pair cache continuing the stream
// where the draws ended) and the cast into the image.  One warp per stamp.
template <typename T>
__global__ void __launch_bounds__(kNoiseWarps * 32) finish_kernel(const __grid_constant__ NoiseArgs a)
{
    __shared__ uint32_t state[kNoiseWarps][kMtN];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kNoiseWarps + warp;
    if (s >= a.n_stamps) return;
    const gsb_noise_stamp sp = a.stamps[s];
    double* w = a.scratch + sp.offset;
    const bool ccd = a.kind == GSB_NOISE_CCD;
    if (ccd && a.p.read_noise > 0.) {
        WarpStream st{state[warp], kMtN, 0, lane};
        mt_seed(st.x, sp.seed, lane);
        st.skip(a.used[s]);
        const double sigma = a.p.gain > 0. ? a.p.read_noise / a.p.gain : a.p.read_noise;
        gaussian_run(st, sp.npix, sigma, [&](long long j, double d) { w[j] += d; });
        if (lane == 0) a.used[s] = st.used;
    }
    __syncwarp();
    T* img = pix_ptr<T>(a.image, sp.offset);
    for (long long j = lane; j < sp.npix; j += 32) img[j] = finish_pixel<T>(w[j], a.p);
}

template <typename T>
int launch_noise(const NoiseArgs& a, int max_npix, cudaStream_t stream)
{
    const int warp_grid = (a.n_stamps + kNoiseWarps - 1) / kNoiseWarps;
    if (a.kind == GSB_NOISE_GAUSSIAN || a.kind == GSB_NOISE_VARIABLE_GAUSSIAN || a.kind == GSB_NOISE_UNIFORM) {
        gauss_kernel<T><<<warp_grid, kNoiseWarps * 32, 0, stream>>>(a);
        GSB_CUDA_CHECK(cudaGetLastError());
        return GSB_OK;
    }
    const int chunks = std::max(1, std::min(64, (max_npix + 255) / 256));
    expect_kernel<T><<<dim3(chunks, a.n_stamps), 256, 0, stream>>>(a);
    GSB_CUDA_CHECK(cudaGetLastError());
    poisson_kernel<<<(a.n_stamps + kPoissonWarps - 1) / kPoissonWarps, kPoissonWarps * 32, 0, stream>>>(a);
    GSB_CUDA_CHECK(cudaGetLastError());
    finish_kernel<T><<<warp_grid, kNoiseWarps * 32, 0, stream>>>(a);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

}  // namespace

int add_noise(int kind, const gsb_noise_params* p, const gsb_noise_stamp* d_stamps, int n_stamps,
              int max_npix, void* d_image, int dtype, double* d_scratch, long long* d_used,
              cudaStream_t stream)
{
    if (n_stamps == 0) return GSB_OK;
    NoiseArgs a;
    a.kind = kind;
    a.p = *p;
    a.stamps = d_stamps;
    a.n_stamps = n_stamps;
    a.image = d_image;
    a.dtype = dtype;
    a.scratch = d_scratch;
    a.used = d_used;
    switch (dtype) {
      case GSB_F32: return launch_noise<float>(a, max_npix, stream);
      case GSB_F64: return launch_noise<double>(a, max_npix, stream);
      case GSB_I16: return launch_noise<int16_t>(a, max_npix, stream);
      case GSB_I32: return launch_noise<int32_t>(a, max_npix, stream);
      case GSB_U16: return launch_noise<uint16_t>(a, max_npix, stream);
      case GSB_U32: return launch_noise<uint32_t>(a, max_npix, stream);
    }
    return set_error(GSB_ERR_INVALID, "unknown image dtype");
}

}  // namespace gsb

using namespace gsb;

extern "C" int gsb_add_noise(int kind, const gsb_noise_params* p, const gsb_noise_stamp* d_stamps,
                             int n_stamps, int max_npix, void* d_image, int dtype, double* d_scratch,
                             long long* d_used, void* stream)
{
    if (!p || n_stamps < 0 || (n_stamps > 0 && (!d_stamps || !d_image)))
        return set_error(GSB_ERR_INVALID, "null argument");
    if (kind < GSB_NOISE_GAUSSIAN || kind > GSB_NOISE_UNIFORM)
        return set_error(GSB_ERR_INVALID, "unknown noise kind");
    if (kind == GSB_NOISE_VARIABLE_GAUSSIAN && n_stamps > 0 && !d_scratch)
        return set_error(GSB_ERR_INVALID, "variable Gaussian noise needs the variance of every pixel in d_scratch");
    if (dtype < GSB_F32 || dtype > GSB_U32) return set_error(GSB_ERR_INVALID, "image dtype must be F32, F64, I16, I32, U16 or U32");
    if ((kind == GSB_NOISE_POISSON || kind == GSB_NOISE_CCD) && (!d_scratch || !d_used))
        return set_error(GSB_ERR_INVALID, "Poisson and CCD noise need the FP64 scratch and the draw counts");
    if (max_npix < 0) return set_error(GSB_ERR_INVALID, "negative pixel count");
    if (kind == GSB_NOISE_GAUSSIAN && !(p->sigma >= 0.)) return set_error(GSB_ERR_INVALID, "sigma must be >= 0");
    return add_noise(kind, p, d_stamps, n_stamps, max_npix, d_image, dtype, d_scratch, d_used,
                     (cudaStream_t)stream);
}
