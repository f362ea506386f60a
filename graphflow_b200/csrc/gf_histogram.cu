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
constexpr uint64_t kCoopScratch = 64u + sizeof(CoopHdr) + (1u << 18); // control blocks + up to 1024 CTAs x 64 words

struct DigitClassify {
    static constexpr bool kAlwaysValid = true;
    uint32_t shift;
    GF_D uint32_t operator()(uint32_t k) const { return (k >> shift) & (kHistBins - 1u); }
};

// AND and OR of all values (the digits that vary are the bits of AND ^ OR). A 16-byte-aligned
// array is read as 128-bit words, four per thread in flight; the rest one value at a time.
__global__ void and_or_kernel(const uint32_t* v, uint64_t n, uint32_t* ao)
{
    uint32_t a = 0xFFFFFFFFu, o = 0u;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t scalar_from = 0u;
    if ((reinterpret_cast<uintptr_t>(v) & 15u) == 0u) {
        const uint4* v4 = reinterpret_cast<const uint4*>(v);
        const uint64_t n4 = n / 4u;
        auto take = [&](const uint4 x) {
            a &= x.x & x.y & x.z & x.w;
            o |= x.x | x.y | x.z | x.w;
        };
        uint64_t i = tid;
        for (; i + 3u * stride < n4; i += 4u * stride) {
            const uint4 x0 = __ldg(v4 + i), x1 = __ldg(v4 + i + stride), x2 = __ldg(v4 + i + 2u * stride),
                        x3 = __ldg(v4 + i + 3u * stride);
            take(x0);
            take(x1);
            take(x2);
            take(x3);
        }
        for (; i < n4; i += stride)
            take(__ldg(v4 + i));
        scalar_from = n4 * 4u;
    }
    for (uint64_t i = scalar_from + tid; i < n; i += stride) {
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
// Warp w of block b covers the 512 consecutive values [b kRleBlock + 512 w, + 512) in 16 rounds
// of 32 lanes (coalesced loads); round k's heads are one ballot, so a head's run index is the
// heads before it: the warp's base + the earlier rounds' popcounts + the lower lanes of this round.
constexpr uint32_t kRleRounds = kRleBlock / 256u; // 256 threads = 8 warps x 512 values

// Ballots of the warp's 16 rounds; v[k] = this lane's value of round k.
GF_D void rle_heads(const uint32_t* s, uint64_t n, uint64_t base, uint32_t lane, uint32_t (&mask)[kRleRounds],
                    uint32_t (&v)[kRleRounds])
{
#pragma unroll
    for (uint32_t k = 0; k < kRleRounds; ++k) {
        const uint64_t i = base + 32u * k + lane;
        v[k] = i < n ? s[i] : 0u;
        const bool head = i < n && (i == 0u || v[k] != s[i - 1u]);
        mask[k] = __ballot_sync(0xFFFFFFFFu, head);
    }
}

// Heads before this warp in the block (exclusive over the 8 warps) and the block's total.
GF_D uint32_t rle_block_prefix(uint32_t warp_heads, uint32_t w, uint32_t lane, uint32_t& total)
{
    __shared__ uint32_t ws[8];
    if (lane == 0u)
        ws[w] = warp_heads;
    __syncthreads();
    uint32_t before = 0;
    total = 0;
#pragma unroll
    for (uint32_t i = 0; i < 8u; ++i) {
        before += i < w ? ws[i] : 0u;
        total += ws[i];
    }
    return before;
}

__global__ void __launch_bounds__(256) rle_count_kernel(const uint32_t* s, uint64_t n, uint32_t* block_heads)
{
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t mask[kRleRounds], v[kRleRounds];
    rle_heads(s, n, (uint64_t)blockIdx.x * kRleBlock + 512u * w, lane, mask, v);
    uint32_t c = 0;
#pragma unroll
    for (uint32_t k = 0; k < kRleRounds; ++k)
        c += (uint32_t)__popc(mask[k]);
    uint32_t total = 0;
    rle_block_prefix(c, w, lane, total);
    if (threadIdx.x == 0)
        block_heads[blockIdx.x] = total;
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
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint64_t base = (uint64_t)blockIdx.x * kRleBlock + 512u * w;
    uint32_t mask[kRleRounds], v[kRleRounds];
    rle_heads(s, n, base, lane, mask, v);
    uint32_t c = 0;
#pragma unroll
    for (uint32_t k = 0; k < kRleRounds; ++k)
        c += (uint32_t)__popc(mask[k]);
    uint32_t total = 0;
    uint32_t r = block_base[blockIdx.x] + rle_block_prefix(c, w, lane, total);
    const uint32_t below = (1u << lane) - 1u;
#pragma unroll
    for (uint32_t k = 0; k < kRleRounds; ++k) {
        if ((mask[k] >> lane) & 1u) {
            const uint32_t q = r + (uint32_t)__popc(mask[k] & below);
            row_values[q] = v[k];
            row_start[q] = (uint32_t)(base + 32u * k + lane);
        }
        r += (uint32_t)__popc(mask[k]);
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
        // the pass also writes its chunk table, descriptors and output count (no finish launch)
        e = launch_fused_coop<CoopShape<32>>(s, DigitClassify{shift}, in, out, kHistC, L.region, tiles,
                                                 2u * n_chunks, kHistBins, reserved, (uint32_t)L.R, totals,
                                                 port_chunks, (uint32_t)L.max_k, ctl, kCoopScratch, d_status, sms,
                                                 InlineFinish{table, descs, (uint32_t)L.R, num_out});
        if (e != cudaSuccess)
            return GF_ERR_CUDA;
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
