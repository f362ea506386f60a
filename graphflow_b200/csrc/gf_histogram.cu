// Device histogram of a u32 column: the sorted (value, count) rows that
// examples/particle_feedback/ParticleTypes.hpp:206-219 (histogramOf: sort + run-length encoding)
// computes on the host, here on the GPU.
//
// The sort is a least-significant-digit radix sort whose passes are this library's stable
// partition: each pass partitions the values by one 6-bit digit into 64 ports with the cooperative
// count/plan/scatter kernel (gf_fused_coop.cuh), and the next pass reads the previous pass's output
// chunks in port order. Digits that are the same for every value (found by one AND/OR reduction)
// are skipped. The sorted chunks are gathered into one array and run-length encoded.
#include <algorithm>

#include "gf_fused_coop.cuh"

namespace gf {
namespace {

constexpr uint32_t kHistC = 8192u;    // chunk capacity of the radix passes
constexpr uint32_t kHistTile = 4096u; // keys per tile
constexpr uint32_t kHistBins = 64u;   // 6-bit digits
constexpr uint32_t kRleBlock = 4096u; // values per run-length block (256 threads x 16)
constexpr uint64_t kCoopScratch = 64u + 512u + (1u << 18); // control blocks + up to 1024 CTAs x 64 words

struct DigitClassify {
    static constexpr bool kAlwaysValid = true;
    uint32_t shift;
    GF_D uint32_t operator()(uint32_t k) const { return (k >> shift) & (kHistBins - 1u); }
};

__global__ void and_or_kernel(const uint32_t* v, uint64_t n, uint32_t* ao)
{
    uint32_t a = 0xFFFFFFFFu, o = 0u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        a &= v[i];
        o |= v[i];
    }
    a = __reduce_and_sync(0xFFFFFFFFu, a);
    o = __reduce_or_sync(0xFFFFFFFFu, o);
    if ((threadIdx.x & 31u) == 0u) {
        atomicAnd(ao, a);
        atomicOr(ao + 1, o);
    }
}

__global__ void copy_u32_kernel(const uint32_t* src, uint32_t* dst, uint64_t n)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = src[i];
}

__global__ void hist_iota_kernel(uint32_t* p, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p[i] = i;
}

// Two tiles per chunk: the first pass's contiguous chunks (descs == null), or the previous pass's
// output chunks in their published (port) order; chunks beyond the count get empty tiles.
__global__ void hist_tiles_kernel(uint64_t n, uint32_t n_chunks, const gf_out_desc* descs, const uint32_t* num_out,
                                  gf_tile* tiles)
{
    for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < n_chunks; f += gridDim.x * blockDim.x) {
        uint32_t chunk = 0, fill = 0;
        if (descs == nullptr) {
            chunk = f;
            const uint64_t left = n - (uint64_t)f * kHistC;
            fill = (uint32_t)(left < kHistC ? left : kHistC);
        } else if (f < *num_out) {
            chunk = descs[f].chunk_index;
            fill = descs[f].fill;
        }
        tiles[2u * f] = gf_tile{chunk, 0u, fill < kHistTile ? fill : kHistTile};
        tiles[2u * f + 1u] = gf_tile{chunk, kHistTile, fill > kHistTile ? fill - kHistTile : 0u};
    }
}

// offsets[f] = sum of the fills of chunks 0..f-1 in published order (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) hist_offsets_kernel(const gf_out_desc* descs, const uint32_t* num_out,
                                                            uint32_t* offsets)
{
    __shared__ uint32_t warp_sum[32];
    const uint32_t r = *num_out, lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < r; base += 1024u) {
        const uint32_t f = base + threadIdx.x;
        const uint32_t x = f < r ? descs[f].fill : 0u;
        uint32_t incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if ((int)lane >= o)
                incl += y;
        }
        if (lane == 31u)
            warp_sum[w] = incl;
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t i = 0; i < 32u; ++i) {
            before += i < w ? warp_sum[i] : 0u;
            total += warp_sum[i];
        }
        if (f < r)
            offsets[f] = carry + before + incl - x;
        carry += total;
        __syncthreads();
    }
}

// Gathers the published chunks, in order, into one contiguous array.
__global__ void hist_gather_kernel(const uint32_t* src, const gf_out_desc* descs, const uint32_t* num_out,
                                   const uint32_t* offsets, uint32_t* dst)
{
    for (uint32_t f = blockIdx.x; f < *num_out; f += gridDim.x) {
        const gf_out_desc d = descs[f];
        const uint32_t* s = src + (uint64_t)d.chunk_index * kHistC;
        uint32_t* t = dst + offsets[f];
        for (uint32_t i = threadIdx.x; i < d.fill; i += blockDim.x)
            t[i] = s[i];
    }
}

// Run-length encoding of a sorted array: a run starts at i = 0 and wherever s[i] != s[i - 1].
GF_D uint32_t heads_of_thread(const uint32_t* s, uint64_t n, uint64_t first, uint32_t (&flag)[16])
{
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const uint64_t i = first + (uint64_t)k;
        flag[k] = (i < n && (i == 0u || s[i] != s[i - 1u])) ? 1u : 0u;
        c += flag[k];
    }
    return c;
}

__global__ void __launch_bounds__(256) rle_count_kernel(const uint32_t* s, uint64_t n, uint32_t* block_heads)
{
    uint32_t flag[16];
    const uint64_t first = (uint64_t)blockIdx.x * kRleBlock + 16u * threadIdx.x;
    uint32_t c = heads_of_thread(s, n, first, flag);
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    __shared__ uint32_t ws[8];
    if ((threadIdx.x & 31u) == 0u)
        ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < 8; ++i)
            t += ws[i];
        block_heads[blockIdx.x] = t;
    }
}

// Exclusive scan of the per-block head counts in place; *num_rows = the total (one CTA).
__global__ void __launch_bounds__(1024) rle_scan_kernel(uint32_t* block_heads, uint32_t nb, uint32_t* num_rows)
{
    __shared__ uint32_t warp_sum[32];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += 1024u) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t x = i < nb ? block_heads[i] : 0u;
        uint32_t incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if ((int)lane >= o)
                incl += y;
        }
        if (lane == 31u)
            warp_sum[w] = incl;
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t k = 0; k < 32u; ++k) {
            before += k < w ? warp_sum[k] : 0u;
            total += warp_sum[k];
        }
        if (i < nb)
            block_heads[i] = carry + before + incl - x;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *num_rows = carry;
}

// Writes each run's value and start position in run order.
__global__ void __launch_bounds__(256) rle_write_kernel(const uint32_t* s, uint64_t n, const uint32_t* block_base,
                                                        uint32_t* row_values, uint32_t* row_start)
{
    uint32_t flag[16];
    const uint64_t first = (uint64_t)blockIdx.x * kRleBlock + 16u * threadIdx.x;
    const uint32_t c = heads_of_thread(s, n, first, flag);
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((int)lane >= o)
            incl += y;
    }
    __shared__ uint32_t ws[8];
    if (lane == 31u)
        ws[w] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t i = 0; i < w; ++i)
        before += ws[i];
    uint32_t r = block_base[blockIdx.x] + before + incl - c;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        if (flag[k]) {
            row_values[r] = s[first + k];
            row_start[r] = (uint32_t)(first + k);
            ++r;
        }
    }
}

__global__ void rle_counts_kernel(const uint32_t* row_start, const uint32_t* num_rows, uint64_t n,
                                  unsigned long long* row_counts)
{
    const uint32_t rows = *num_rows;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const uint64_t end = r + 1u < rows ? row_start[r + 1u] : n;
        row_counts[r] = end - row_start[r];
    }
}

struct HistLayout {
    uint64_t n, n_in, R, region, tiles, max_k;
    uint64_t x, y, tile, reserved, ctl, totals, port_chunks, table, descs, num_out, offsets, ao, block_heads, total;
    explicit HistLayout(uint64_t n_) : n(n_)
    {
        n_in = (n + kHistC - 1u) / kHistC;
        R = std::min<uint64_t>(n, n_in + kHistBins - 1u); // outputChunkBound(n, C, 64)
        region = std::max<uint64_t>(R, n_in) * kHistC;
        tiles = 2u * std::max<uint64_t>(std::max<uint64_t>(n_in, R), 1u);
        max_k = std::max<uint64_t>(n_in, 1u);
        auto up = [](uint64_t v) { return (v + 255u) & ~uint64_t(255u); };
        uint64_t o = 0;
        x = o;
        o += up(region * 4u);
        y = o;
        o += up(region * 4u);
        tile = o;
        o += up(tiles * sizeof(gf_tile));
        reserved = o;
        o += up(std::max<uint64_t>(R, 1u) * 4u);
        ctl = o;
        o += up(kCoopScratch);
        totals = o;
        o += up(kHistBins * 4u);
        port_chunks = o;
        o += up(kHistBins * max_k * 8u);
        table = o;
        o += up((kHistBins + std::max<uint64_t>(R, 1u)) * 4u);
        descs = o;
        o += up(std::max<uint64_t>(R, 1u) * sizeof(gf_out_desc));
        num_out = o;
        o += 256u;
        offsets = o;
        o += up((std::max<uint64_t>(R, 1u) + 1u) * 4u);
        ao = o;
        o += 256u;
        block_heads = o;
        o += up(((n + kRleBlock - 1u) / kRleBlock + 1u) * 4u);
        total = o;
    }
};

} // namespace
} // namespace gf

using namespace gf;

extern "C" {

gf_status gf_histogram_scratch_bytes(uint64_t n, uint64_t* h_bytes)
{
    if (h_bytes == nullptr || n > 0x80000000ull)
        return GF_ERR_ARGUMENT;
    *h_bytes = HistLayout(n).total;
    return GF_OK;
}

gf_status gf_histogram_u32(void* stream, const uint32_t* d_values, uint64_t n, void* d_scratch,
                           uint64_t scratch_bytes, uint32_t* d_row_values, unsigned long long* d_row_counts,
                           uint32_t* d_num_rows, uint32_t* d_status)
{
    if (n > 0x80000000ull || d_num_rows == nullptr || d_status == nullptr || d_scratch == nullptr ||
        (reinterpret_cast<uintptr_t>(d_scratch) & 255u) != 0u ||
        (n != 0u && (d_values == nullptr || d_row_values == nullptr || d_row_counts == nullptr)))
        return GF_ERR_ARGUMENT;
    const HistLayout L(n);
    if (scratch_bytes < L.total)
        return GF_ERR_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    auto cuda_ok = [](cudaError_t e) { return e == cudaSuccess ? GF_OK : GF_ERR_CUDA; };
    if (n == 0u)
        return cuda_ok(cudaMemsetAsync(d_num_rows, 0, 4u, s));
    char* base = static_cast<char*>(d_scratch);
    auto* X = reinterpret_cast<uint32_t*>(base + L.x);
    auto* Y = reinterpret_cast<uint32_t*>(base + L.y);
    auto* tiles = reinterpret_cast<gf_tile*>(base + L.tile);
    auto* reserved = reinterpret_cast<uint32_t*>(base + L.reserved);
    auto* ctl = reinterpret_cast<FusedCtl*>(base + L.ctl);
    auto* totals = reinterpret_cast<uint32_t*>(base + L.totals);
    auto* port_chunks = reinterpret_cast<unsigned long long*>(base + L.port_chunks);
    auto* table = reinterpret_cast<uint32_t*>(base + L.table);
    auto* descs = reinterpret_cast<gf_out_desc*>(base + L.descs);
    auto* num_out = reinterpret_cast<uint32_t*>(base + L.num_out);
    auto* offsets = reinterpret_cast<uint32_t*>(base + L.offsets);
    auto* ao = reinterpret_cast<uint32_t*>(base + L.ao);
    auto* block_heads = reinterpret_cast<uint32_t*>(base + L.block_heads);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned g = (unsigned)std::min<uint64_t>((n + 255u) / 256u, (uint64_t)sms * 8u);

    // which digits vary: one AND/OR reduction, read on the host (the one wait of this call)
    const uint32_t ao_init[2] = {0xFFFFFFFFu, 0u};
    cudaError_t e = cudaMemcpyAsync(ao, ao_init, 8u, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return GF_ERR_CUDA;
    and_or_kernel<<<g, 256, 0, s>>>(d_values, n, ao);
    uint32_t h_ao[2] = {0u, 0u};
    e = cudaMemcpyAsync(h_ao, ao, 8u, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return GF_ERR_CUDA;
    const uint32_t varying = h_ao[0] ^ h_ao[1];

    const uint32_t* sorted = d_values; // every value equal: already sorted
    uint32_t* spare = X;
    bool any = false;
    uint32_t* in = Y; // each pass reads `in` and writes `out`; they swap after every pass
    uint32_t* out = X;
    for (uint32_t shift = 0; shift < 32u; shift += 6u) {
        if (((varying >> shift) & (kHistBins - 1u)) == 0u)
            continue;
        if (!any) { // the first pass reads a padded copy of the values in chunk layout
            copy_u32_kernel<<<g, 256, 0, s>>>(d_values, Y, n);
            hist_iota_kernel<<<(unsigned)((L.R + 255u) / 256u), 256, 0, s>>>(reserved, (uint32_t)L.R);
            e = cudaMemsetAsync(ctl, 0, sizeof(FusedCtl), s);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(port_chunks, 0, kHistBins * L.max_k * 8u, s);
            if (e != cudaSuccess)
                return GF_ERR_CUDA;
        }
        const uint32_t n_chunks = any ? (uint32_t)L.R : (uint32_t)L.n_in;
        hist_tiles_kernel<<<(n_chunks + 255u) / 256u, 256, 0, s>>>(n, n_chunks, any ? descs : nullptr, num_out,
                                                                   tiles);
        e = launch_fused_coop<CoopShape<32>>(s, DigitClassify{shift}, in, out, kHistC, L.region, tiles,
                                                 2u * n_chunks, kHistBins, reserved, (uint32_t)L.R, totals,
                                                 port_chunks, (uint32_t)L.max_k, ctl, kCoopScratch, d_status, sms);
        if (e != cudaSuccess)
            return GF_ERR_CUDA;
        constexpr int FT = 1024;
        const size_t fsmem = sizeof(uint32_t) * (4096u * 2u + FT / 32 + 1);
        e = cudaFuncSetAttribute(fused_finish_kernel<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsmem);
        if (e != cudaSuccess)
            return GF_ERR_CUDA;
        fused_finish_kernel<FT><<<1, FT, fsmem, s>>>(totals, port_chunks, kHistBins, kHistC, FastDiv(kHistC),
                                                      (uint32_t)L.max_k, ctl, table, descs, (uint32_t)L.R, num_out,
                                                      d_status);
        any = true;
        std::swap(in, out); // the next pass reads this pass's output region
    }
    if (any) { // `in` holds the last pass's output chunks; gather them into the other region
        uint32_t* dst = out; // the region the last pass read
        hist_offsets_kernel<<<1, 1024, 0, s>>>(descs, num_out, offsets);
        hist_gather_kernel<<<(unsigned)std::min<uint64_t>(L.R, 65535u), 256, 0, s>>>(in, descs, num_out, offsets, dst);
        sorted = dst;
        spare = in;
    }
    const uint32_t nb = (uint32_t)((n + kRleBlock - 1u) / kRleBlock);
    rle_count_kernel<<<nb, 256, 0, s>>>(sorted, n, block_heads);
    rle_scan_kernel<<<1, 1024, 0, s>>>(block_heads, nb, d_num_rows);
    rle_write_kernel<<<nb, 256, 0, s>>>(sorted, n, block_heads, d_row_values, spare);
    rle_counts_kernel<<<g, 256, 0, s>>>(spare, d_num_rows, n, d_row_counts);
    return cuda_ok(cudaGetLastError());
}

} // extern "C"
