// FITS file images of stamp batches, assembled on the device (the format of galsim/fits.py
// writeMulti / writeCube, FITS Standard 4.0): each HDU is its header (80-byte cards, already
// formatted on the host and padded to 2880-byte blocks) followed by its pixels in big-endian
// order, zero-padded to a block.  One launch writes every HDU of the file into one buffer, which
// then leaves the device with one copy.
//
// Layout of the work: grid.x walks the HDUs, grid.y the 4 KB chunks of one HDU (grid-stride), so
// a file of thousands of small stamps and a data cube of one large HDU both fill the SMs.
// Headers and padding move as 16-byte words (every HDU starts on a 2880-byte boundary, a
// multiple of 16); pixels are read in the stamp buffer's own order and stored byte-swapped.
#include <algorithm>

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

// W: the pixel word (4 or 8 bytes).
template <class W>
__global__ void __launch_bounds__(kFitsThreads) fits_pack_kernel(const gsb_fits_hdu* hdus,
                                                                 const unsigned char* headers,
                                                                 const W* src, unsigned char* out)
{
    const gsb_fits_hdu h = hdus[blockIdx.x];
    unsigned char* dst = out + h.dst;
    // header: 16-byte words
    const uint4* hs = reinterpret_cast<const uint4*>(headers + h.header_src);
    uint4* hd = reinterpret_cast<uint4*>(dst);
    const long long hwords = h.header_len / 16;
    const long long step = (long long)gridDim.y * kFitsThreads;
    for (long long w = (long long)blockIdx.y * kFitsThreads + threadIdx.x; w < hwords; w += step)
        hd[w] = hs[w];
    // pixels
    W* pd = reinterpret_cast<W*>(dst + h.header_len);
    const W* ps = src + h.data_src;
    for (long long e = (long long)blockIdx.y * kFitsThreads + threadIdx.x; e < h.n_elem; e += step)
        pd[e] = bswap<W>(ps[e]);
    // zero padding up to the next block, in bytes (at most 2879)
    const long long dbytes = h.n_elem * (long long)sizeof(W);
    const long long pad = (kFitsBlock - dbytes % kFitsBlock) % kFitsBlock;
    unsigned char* pz = dst + h.header_len + dbytes;
    for (long long b = (long long)blockIdx.y * kFitsThreads + threadIdx.x; b < pad; b += step)
        pz[b] = 0;
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
    long long max_chunks = 1;
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
        max_chunks = std::max<long long>(max_chunks, (units + kFitsThreads - 1) / kFitsThreads);
    }
    const unsigned gy = (unsigned)std::min<long long>(max_chunks, 1024);
    gsb_fits_hdu* d_hdus = nullptr;
    GSB_CUDA_CHECK(cudaMallocAsync(&d_hdus, sizeof(gsb_fits_hdu) * n_hdus, stream));
    GSB_CUDA_CHECK(cudaMemcpyAsync(d_hdus, h_hdus, sizeof(gsb_fits_hdu) * n_hdus, cudaMemcpyHostToDevice, stream));
    const dim3 grid((unsigned)n_hdus, gy);
    if (dtype == GSB_F32)
        fits_pack_kernel<unsigned int><<<grid, kFitsThreads, 0, stream>>>(
            d_hdus, static_cast<const unsigned char*>(d_headers), static_cast<const unsigned int*>(d_src),
            static_cast<unsigned char*>(d_out));
    else
        fits_pack_kernel<unsigned long long><<<grid, kFitsThreads, 0, stream>>>(
            d_hdus, static_cast<const unsigned char*>(d_headers), static_cast<const unsigned long long*>(d_src),
            static_cast<unsigned char*>(d_out));
    GSB_CUDA_CHECK(cudaGetLastError());
    GSB_CUDA_CHECK(cudaFreeAsync(d_hdus, stream));
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
