// FITS file images of stamp batches, assembled on the device (the format of galsim/fits.py
// writeMulti / writeCube, FITS Standard 4.0): each HDU is its header (80-byte cards, already
// formatted on the host and padded to 2880-byte blocks) followed by its pixels in big-endian
// order, zero-padded to a block.  One launch writes every HDU of the file into one buffer, which
// then leaves the device with one copy.
//
// Layout of the work: one block per chunk of 256 units (16-byte header words, pixels, padding
// bytes) of one HDU, so a file of thousands of small stamps and a data cube of one large HDU
// both fill the SMs with as many blocks as their bytes need.
// Headers and padding move as 16-byte words (every HDU starts on a 2880-byte boundary, a
// multiple of 16); pixels are read in the stamp buffer's own order and stored byte-swapped.
#include <algorithm>
#include <vector>

#include "gsb_internal.cuh"

namespace gsb {

namespace {

constexpr long long kFitsBlock = 2880;
constexpr int kFitsThreads = 256;

__device__ __forceinline__ unsigned int bswap32(unsigned int v) { return __byte_perm(v, 0, 0x0123); }

template <class W>
__device__ __forceinline__ W bswap(W v);

template <>
__device__ __forceinline__ unsigned int bswap<unsigned int>(unsigned int v) { return bswap32(v); }

template <>
__device__ __forceinline__ unsigned long long bswap<unsigned long long>(unsigned long long v)
{
    const unsigned int lo = (unsigned int)v, hi = (unsigned int)(v >> 32);
    return ((unsigned long long)bswap32(lo) << 32) | bswap32(hi);
}

// W: the pixel word (4 or 8 bytes).  One block per chunk of kFitsThreads units of one HDU: the
// blocks of HDU h are chunk_base[h] .. chunk_base[h + 1] - 1 (host prefix sums), found by a
// binary search, so a small stamp costs as few blocks as its size needs.
template <class W>
__global__ void __launch_bounds__(kFitsThreads) fits_pack_kernel(const gsb_fits_hdu* hdus,
                                                                 const long long* chunk_base, int n_hdus,
                                                                 const unsigned char* headers,
                                                                 const W* src, unsigned char* out)
{
    const long long blk = blockIdx.x;
    int lo = 0, hi = n_hdus - 1;               // the last h with chunk_base[h] <= blk
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (chunk_base[mid] <= blk) lo = mid; else hi = mid - 1;
    }
    const gsb_fits_hdu h = hdus[lo];
    const long long u = (blk - chunk_base[lo]) * kFitsThreads + threadIdx.x;   // unit index
    unsigned char* dst = out + h.dst;
    // header: 16-byte words
    if (u < h.header_len / 16)
        reinterpret_cast<uint4*>(dst)[u] = reinterpret_cast<const uint4*>(headers + h.header_src)[u];
    // pixels
    if (u < h.n_elem)
        reinterpret_cast<W*>(dst + h.header_len)[u] = bswap<W>(src[h.data_src + u]);
    // zero padding up to the next block, in bytes (at most 2879)
    const long long dbytes = h.n_elem * (long long)sizeof(W);
    const long long pad = (kFitsBlock - dbytes % kFitsBlock) % kFitsBlock;
    if (u < pad) dst[h.header_len + dbytes + u] = 0;
}

}  // namespace

int fits_pack(const gsb_fits_hdu* h_hdus, int n_hdus, const void* d_headers, long long header_bytes,
              const void* d_src, long long src_elems, int dtype, void* d_out, long long out_bytes,
              cudaStream_t stream)
{
    if (n_hdus < 0 || (n_hdus > 0 && (!h_hdus || !d_headers || !d_src || !d_out)))
        return set_error(GSB_ERR_INVALID, "gsb_fits_pack: null pointer or negative count");
    if (dtype != GSB_F32 && dtype != GSB_F64) return set_error(GSB_ERR_INVALID, "gsb_fits_pack: dtype");
    if (n_hdus == 0) return GSB_OK;
    if (reinterpret_cast<uintptr_t>(d_headers) % 16 || reinterpret_cast<uintptr_t>(d_out) % 16)
        return set_error(GSB_ERR_INVALID, "gsb_fits_pack: header and output buffers must be 16-byte aligned");
    const long long esz = dtype == GSB_F32 ? 4 : 8;
    if (reinterpret_cast<uintptr_t>(d_src) % esz)
        return set_error(GSB_ERR_INVALID, "gsb_fits_pack: misaligned pixel buffer");
    // Every record must stay inside its buffers, start on a block, and not overlap the next HDU.
    std::vector<long long> chunk_base(n_hdus + 1, 0);
    for (int i = 0; i < n_hdus; ++i) {
        const gsb_fits_hdu& h = h_hdus[i];
        const long long dbytes = h.n_elem * esz;
        const long long total = h.header_len + (dbytes + kFitsBlock - 1) / kFitsBlock * kFitsBlock;
        if (h.header_src < 0 || h.header_len <= 0 || h.header_len % kFitsBlock || h.header_src % 16 ||
            h.header_src + h.header_len > header_bytes || h.n_elem < 0 || h.data_src < 0 ||
            h.data_src + h.n_elem > src_elems || h.dst < 0 || h.dst % kFitsBlock || h.dst + total > out_bytes)
            return set_error(GSB_ERR_INVALID, "gsb_fits_pack: HDU record out of range or misaligned");
        if (i + 1 < n_hdus && h_hdus[i + 1].dst < h.dst + total)
            return set_error(GSB_ERR_INVALID, "gsb_fits_pack: HDUs must follow one another without overlap");
        const long long units = std::max<long long>(h.header_len / 16, std::max<long long>(h.n_elem, kFitsBlock));
        chunk_base[i + 1] = chunk_base[i] + (units + kFitsThreads - 1) / kFitsThreads;
    }
    const long long blocks = chunk_base[n_hdus];
    if (blocks > 2147483647LL) return set_error(GSB_ERR_INVALID, "gsb_fits_pack: file image too large");
    gsb_fits_hdu* d_hdus = nullptr;
    long long* d_base = nullptr;
    GSB_CUDA_CHECK(cudaMallocAsync(&d_hdus, sizeof(gsb_fits_hdu) * n_hdus, stream));
    GSB_CUDA_CHECK(cudaMallocAsync(&d_base, sizeof(long long) * (n_hdus + 1), stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(d_hdus, h_hdus, sizeof(gsb_fits_hdu) * n_hdus, cudaMemcpyHostToDevice, stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(d_base, chunk_base.data(), sizeof(long long) * (n_hdus + 1),
                                   cudaMemcpyHostToDevice, stream));
    if (dtype == GSB_F32)
        fits_pack_kernel<unsigned int><<<(unsigned)blocks, kFitsThreads, 0, stream>>>(
            d_hdus, d_base, n_hdus, static_cast<const unsigned char*>(d_headers),
            static_cast<const unsigned int*>(d_src), static_cast<unsigned char*>(d_out));
    else
        fits_pack_kernel<unsigned long long><<<(unsigned)blocks, kFitsThreads, 0, stream>>>(
            d_hdus, d_base, n_hdus, static_cast<const unsigned char*>(d_headers),
            static_cast<const unsigned long long*>(d_src), static_cast<unsigned char*>(d_out));
    GSB_CUDA_CHECK(cudaGetLastError());
    GSB_CUDA_CHECK(cudaFreeAsync(d_hdus, stream));
    GSB_CUDA_CHECK(cudaFreeAsync(d_base, stream));
    return GSB_OK;
}

}  // namespace gsb

extern "C" int gsb_fits_pack(const gsb_fits_hdu* h_hdus, int n_hdus, const void* d_headers,
                             long long header_bytes, const void* d_src, long long src_elems, int dtype,
                             void* d_out, long long out_bytes, void* stream)
{
    return gsb::fits_pack(h_hdus, n_hdus, d_headers, header_bytes, d_src, src_elems, dtype, d_out,
                          out_bytes, static_cast<cudaStream_t>(stream));
}
