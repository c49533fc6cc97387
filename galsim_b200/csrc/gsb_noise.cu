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
// One warp per stamp.  The warp holds the 624-word state in shared memory and regenerates it
// cooperatively (the twist in 32-word chunks, whose dependences span 227 and 397 words).
// Gaussian pairs are independent once their two words are known, so the lanes take consecutive
// pairs of each block; Poisson draws consume a data-dependent number of words, so the warp
// runs them in lockstep (every lane computes the same draw) and only the twists are shared.
#include <cuda_runtime.h>
#include <stdint.h>

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

// BaseDeviate(seed): mt11213b(seed), two draws discarded, the third seeds the mt19937
// (lane 0 runs the sequential recurrences; the result is left in x with the position at the
// end of the block, i.e. the first draw twists).
__device__ void mt_seed(uint32_t* x, long long seed, int lane)
{
    if (lane == 0) {
        // mt11213b: w 32, n 351, m 175, r 19, a 0xccab8ee7, tempering (11, 7 0x31b6ab00,
        // 15 0xffe50000, 17)
        constexpr int n = 351, m = 175;
        uint32_t* a = x;     // the first 351 words of the buffer serve as its state
        a[0] = uint32_t(seed);
        for (int i = 1; i < n; ++i) a[i] = 1812433253u * (a[i - 1] ^ (a[i - 1] >> 30)) + uint32_t(i);
        uint32_t out = 0;
        for (int k = 0; k < 3; ++k) {    // draws 0 and 1 are discarded
            // only the first three words are needed after the twist: x'[k] = x[k+m] ^ mix(x[k], x[k+1])
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
    __syncwarp();
}

// A warp's position in its stream: the state x (shared), the index i of the next word in the
// current block (kMtN = exhausted), and the count of words consumed since seeding.
struct WarpStream {
    uint32_t* x;
    int i;
    long long used;
    int lane;

    __device__ uint32_t next()           // every lane calls, all get the same word
    {
        if (i == kMtN) { mt_twist(x, lane); i = 0; }
        const uint32_t w = mt_temper(x[i]);
        ++i;
        ++used;
        return w;
    }
    __device__ double uniform() { return double(next()) * (1. / 4294967296.); }
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

// log k! for k < 10 (the table PTRD uses below the Stirling branch).
__device__ __forceinline__ double log_factorial_small(int k)
{
    double r = 0.;
    for (int i = 2; i <= k; ++i) r += log(double(i));
    return r;
}

// One Poisson draw with the warp's stream (all lanes in lockstep).
__device__ double poisson_draw(WarpStream& st, double mean)
{
    if (mean < 10.) {
        double p = exp(-mean);
        double x = 0.;
        double u = st.uniform();
        // ends once the cumulative probability reaches u <= 1 - 2^-32 (x well below 100 for
        // mean < 10); the bound only guards against a non-finite mean
        while (u > p && x < 1000.) {
            u = u - p;
            x += 1.;
            p = mean * p / x;
        }
        return x;
    }
    const double smu = sqrt(mean);
    const double b = 0.931 + 2.53 * smu;
    const double a = -0.059 + 0.02483 * b;
    const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
    const double v_r = 0.9277 - 3.6224 / (b - 2);
    for (int iter = 0; iter < (1 << 20); ++iter) {
        double u;
        double v = st.uniform();
        if (v <= 0.86 * v_r) {
            u = v / v_r - 0.43;
            return floor((2 * a / (0.5 - fabs(u)) + b) * u + mean + 0.445);
        }
        if (v >= v_r) {
            u = st.uniform() - 0.5;
        } else {
            u = v / v_r - 0.93;
            u = ((u < 0) ? -0.5 : 0.5) - u;
            v = st.uniform() * v_r;
        }
        const double us = 0.5 - fabs(u);
        if (us < 0.013 && v > us) continue;
        const double k = floor((2 * a / us + b) * u + mean + 0.445);
        v = v * inv_alpha / (a / (us * us) + b);
        const double log_sqrt_2pi = 0.91893853320467267;
        if (k >= 10) {
            if (log(v * smu) <= (k + 0.5) * log(mean / k) - mean - log_sqrt_2pi + k -
                                    (1 / 12. - (1 / 360. - 1 / (1260. * k * k)) / (k * k)) / k)
                return k;
        } else if (k >= 0) {
            if (log(v) <= k * log(mean) - mean - log_factorial_small(int(k))) return k;
        }
    }
    return mean;   // unreachable in practice: the rejection loop accepts with probability > 0.8
}

struct NoiseArgs {
    int kind;
    gsb_noise_params p;
    const gsb_noise_stamp* stamps;
    int n_stamps;
    void* image;
    int dtype;
    double* scratch;       // FP64 value per pixel (Poisson / CCD), indexed like the image
    long long* used;
};

// The cast back into the image and the sky bookkeeping of PoissonNoise / CCDNoise._applyTo:
// frac_sky is subtracted in FP64 before the cast, int_sky after it (in the image type when the
// caller's int_sky has the image's type, as Image.__isub__ does).
template <typename T>
__device__ __forceinline__ T finish_pixel(double w, const gsb_noise_params& p)
{
    if (p.frac_sky != 0.) w -= p.frac_sky;
    T out = T(w);
    if (p.int_sky != 0.) out = p.int_sky_same_dtype ? T(out - T(p.int_sky)) : T(double(out) - p.int_sky);
    return out;
}

template <typename T>
__device__ void noise_stamp(const NoiseArgs& a, const gsb_noise_stamp& sp, WarpStream& st)
{
    T* img = pix_ptr<T>(a.image, sp.offset);
    const long long n = sp.npix;
    const int lane = st.lane;
    if (a.kind == GSB_NOISE_GAUSSIAN) {
        gaussian_run(st, n, a.p.sigma, [&](long long j, double d) { img[j] = img[j] + T(d); });
        return;
    }
    double* w = a.scratch + sp.offset;
    const bool ccd = a.kind == GSB_NOISE_CCD;
    const double gain = ccd ? a.p.gain : 1.;
    // expectation per pixel (all lanes)
    for (long long j = lane; j < n; j += 32) {
        double v = double(img[j]);
        if (a.p.sky_level != 0.) v += a.p.sky_level;
        if (!ccd || gain > 0.) {
            if (ccd) v *= gain;
            if (v < 0.) v = 0.;
        }
        w[j] = v;
    }
    __syncwarp();
    if (!ccd || gain > 0.) {
        // the draws in pixel order, every lane computing the same value (PoissonDeviate
        // generateFromExpectation with its mean switching; the normal branch above 2^30 keeps
        // its pair cache while the mean is unchanged)
        double cur_mean = 1.;
        bool use_gd = false, gd_valid = false;
        double gd_rho = 0., gd_r1 = 0.;
        const double kMaxPoisson = double(1 << 30);
        for (long long j = 0; j < n; ++j) {
            double v = w[j];
            if (v > 0.) {
                if (v != cur_mean) {
                    cur_mean = v;
                    if (v > kMaxPoisson) {
                        use_gd = true;
                    } else {
                        use_gd = false;
                        gd_valid = false;
                    }
                }
                if (use_gd) {
                    const double sg = sqrt(v);
                    if (!gd_valid) {
                        gd_r1 = st.uniform();
                        const double r2 = st.uniform();
                        gd_rho = sqrt(-2. * log(1. - r2));
                        gd_valid = true;
                        v = gd_rho * cos(kPi2 * gd_r1) * sg + v;
                    } else {
                        gd_valid = false;
                        v = gd_rho * sin(kPi2 * gd_r1) * sg + v;
                    }
                } else {
                    v = poisson_draw(st, v);
                }
            }
            if (ccd) v /= gain;
            __syncwarp();
            if (lane == 0) w[j] = v;
            __syncwarp();
        }
    }
    if (ccd && a.p.read_noise > 0.) {
        const double sigma = gain > 0. ? a.p.read_noise / gain : a.p.read_noise;
        gaussian_run(st, n, sigma, [&](long long j, double d) { w[j] += d; });
    }
    __syncwarp();
    for (long long j = lane; j < n; j += 32) img[j] = finish_pixel<T>(w[j], a.p);
}

__global__ void __launch_bounds__(kNoiseWarps * 32) noise_kernel(const __grid_constant__ NoiseArgs a)
{
    __shared__ uint32_t state[kNoiseWarps][kMtN];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kNoiseWarps + warp;
    if (s >= a.n_stamps) return;
    const gsb_noise_stamp sp = a.stamps[s];
    WarpStream st{state[warp], kMtN, 0, lane};
    mt_seed(st.x, sp.seed, lane);
    st.skip(sp.skip);
    if (a.dtype == GSB_F32) noise_stamp<float>(a, sp, st);
    else noise_stamp<double>(a, sp, st);
    if (lane == 0 && a.used) a.used[s] = st.used;     // words consumed since seeding
}

}  // namespace

int add_noise(int kind, const gsb_noise_params* p, const gsb_noise_stamp* d_stamps, int n_stamps,
              void* d_image, int dtype, double* d_scratch, long long* d_used, cudaStream_t stream)
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
    const int grid = (n_stamps + kNoiseWarps - 1) / kNoiseWarps;
    noise_kernel<<<grid, kNoiseWarps * 32, 0, stream>>>(a);
    GSB_CUDA_CHECK(cudaGetLastError());
    return GSB_OK;
}

}  // namespace gsb

using namespace gsb;

extern "C" int gsb_add_noise(int kind, const gsb_noise_params* p, const gsb_noise_stamp* d_stamps,
                             int n_stamps, void* d_image, int dtype, double* d_scratch,
                             long long* d_used, void* stream)
{
    if (!p || n_stamps < 0 || (n_stamps > 0 && (!d_stamps || !d_image)))
        return set_error(GSB_ERR_INVALID, "null argument");
    if (kind < GSB_NOISE_GAUSSIAN || kind > GSB_NOISE_CCD)
        return set_error(GSB_ERR_INVALID, "unknown noise kind");
    if (dtype != GSB_F32 && dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "image dtype must be F32 or F64");
    if (kind != GSB_NOISE_GAUSSIAN && !d_scratch)
        return set_error(GSB_ERR_INVALID, "Poisson and CCD noise need the FP64 scratch buffer");
    if (kind == GSB_NOISE_GAUSSIAN && !(p->sigma >= 0.)) return set_error(GSB_ERR_INVALID, "sigma must be >= 0");
    return add_noise(kind, p, d_stamps, n_stamps, d_image, dtype, d_scratch, d_used, (cudaStream_t)stream);
}
