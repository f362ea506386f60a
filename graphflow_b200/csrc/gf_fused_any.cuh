// Cooperative fused partition for any payload, classifier and updater (up to 64 ports): the
// count -> grid barrier -> plan -> scatter design of fused_partition_coop_kernel
// (gf_fused_coop.cuh) over the front end's access policies, for whole-list batches of the
// device-resident runs. Same contract as fused_partition_kernel with an inline finish (per-port
// totals, the reference's dense plan and table, graph/DenseBinTable.hpp:39-91, the output
// descriptors), every port's particles in input order, and no per-tile look-back:
//   phase 1  CTA c owns the contiguous tiles [n c / G, n (c + 1) / G); it loads and classifies
//            every particle once, keeps the bin (16 bits per particle, in the scratch) and counts
//            ports in shared memory (warp-aggregated up to 16 ports); its per-port counts go to
//            its row of the scratch and are added to the batch totals;
//   barrier  cooperative launch, bounded wait (coop_grid_barrier);
//   plan     per-port base of this CTA (the rows before it, or the batch total minus the rows
//            after it, whichever is fewer), binBase[b] = sum_{b' < b} ceil(total_b' / C); port b's
//            k-th output chunk is reserved[binBase[b] + k]; the CTAs write the table and the
//            descriptors between them;
//   phase 2  every tile again in order: payloads reloaded, bins from the scratch, a stable rank
//            inside the tile (warp_rank), the updater applied, the tile staged in port order and
//            written out through the plan, the CTA's per-port running bases advanced.
// Traffic per particle: the payload read twice and written once, 2 bytes of bin written and read.
#pragma once

#include "gf_fused_coop.cuh"

namespace gf {
namespace { // internal linkage: see gf_partition.cuh

constexpr uint32_t kAnyCoopMaxBins = 64u;

// Batch totals, the grid-barrier counter and the count of finished CTAs; zeroed before every
// launch (by the launcher, or by the caller's previous launch on the stream).
struct AnyCoopHdr {
    unsigned long long total[kAnyCoopMaxBins];
    unsigned long long done;
    unsigned long long finished;
    unsigned long long pad[6];
};
static_assert(sizeof(AnyCoopHdr) % 64u == 0u, "row alignment");

// Scratch of one launch: header | per-CTA port counts [max_ctas][64] | bins [n_tiles * tile].
inline uint64_t any_coop_scratch_bytes(uint32_t n_tiles, uint32_t tile, uint32_t max_ctas)
{
    return sizeof(AnyCoopHdr) + 4ull * kAnyCoopMaxBins * max_ctas + 2ull * n_tiles * tile + 16u;
}

template <typename Shape, typename P>
constexpr size_t any_coop_smem_bytes(uint32_t B)
{
    return sizeof(P) * Shape::kTile + 4u * Shape::kTile + 4u * Shape::kWarps * B + 4u * (6u * B) +
           4u * (Shape::kWarps + 1u + 8u);
}

template <typename Shape, typename Access, typename Classify, typename Update, typename Post>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) fused_partition_any_coop_kernel(
    Access acc, Classify classify, Update update, uint64_t seed_mixed, uint32_t capacity, FastDiv fdc,
    uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t B, const uint32_t* reserved,
    uint32_t n_reserved, uint32_t* totals, AnyCoopHdr* hdr, uint32_t* cta_cnt, uint16_t* bins16,
    uint32_t* status, InlineFinish fin, Post post)
{
    using P = typename Access::Payload;
    constexpr int T = Shape::kThreads, W = Shape::kWarps, IPT = Shape::kIpt;
    constexpr uint32_t MB = kAnyCoopMaxBins;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* stage = reinterpret_cast<P*>(smem_raw);
    uint32_t* stage_bin = reinterpret_cast<uint32_t*>(stage + Shape::kTile);
    uint32_t* warp_cnt = stage_bin + Shape::kTile;        // [W][B]
    uint32_t* bin_tot = warp_cnt + (size_t)W * B;         // [B]
    uint32_t* bin_excl = bin_tot + B;                     // [B]
    uint32_t* run_base = bin_excl + B;                    // [B] this CTA's next output position per port
    uint32_t* bin_base = run_base + B;                    // [B] first plan chunk of each port
    uint32_t* cnt = bin_base + B;                         // [B] phase 1 counts
    uint32_t* tot = cnt + B;                              // [B] batch totals
    uint32_t* scan_tmp = tot + B;                         // [W + 1]
    uint32_t* misc = scan_tmp + W + 1;                    // [8]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    const uint32_t t_lo = (uint32_t)((uint64_t)n_tiles * c / G), t_hi = (uint32_t)((uint64_t)n_tiles * (c + 1u) / G);

    auto tile_of = [&](uint32_t t, uint64_t& base) -> uint32_t {
        const gf_tile tl = tiles[t];
        base = (uint64_t)tl.chunk_index * capacity + tl.tile_offset;
        const bool ok = tl.count <= (uint32_t)Shape::kTile && base + tl.count <= pool_slots &&
                        tl.tile_offset + tl.count <= capacity;
        if (!ok) {
            if (threadIdx.x == 0)
                set_status(status, GF_INVALID);
            return 0u;
        }
        return tl.count;
    };

    // ---------------- phase 1: classify once, keep the bins, count ports ----------------
    for (uint32_t b = threadIdx.x; b < B; b += T)
        cnt[b] = 0u;
    __syncthreads();
    for (uint32_t t = t_lo; t < t_hi; ++t) {
        uint64_t base = 0;
        const uint32_t count = tile_of(t, base);
        P p[IPT];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            if (i < count)
                p[r] = acc.load(base + i);
        }
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            uint32_t b = kNoBin16;
            if (i < count) {
                const uint32_t v = classify(p[r]);
                if (v < B)
                    b = v;
                else
                    set_status(status, GF_INVALID);
                bins16[(size_t)t * Shape::kTile + i] = (uint16_t)b;
            }
            if (B > 16u) { // many ports: few lanes share one, a plain shared atomic each
                if (b != kNoBin16)
                    atomicAdd(&cnt[b], 1u);
            } else { // few ports: one atomic per distinct port of the warp
                const uint32_t peers = __match_any_sync(0xFFFFFFFFu, b);
                if (b != kNoBin16 && lane == __ffs(peers) - 1)
                    atomicAdd(&cnt[b], (uint32_t)__popc(peers));
            }
        }
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < MB; b += T) {
        const uint32_t v = b < B ? cnt[b] : 0u;
        cta_cnt[(size_t)c * MB + b] = v;
        if (v != 0u)
            atomicAdd(&hdr->total[b], (unsigned long long)v);
    }

    coop_grid_barrier(&hdr->done, status);

    // ---------------- plan ----------------
    const bool before = c <= G - 1u - c;
    for (uint32_t b = threadIdx.x; b < B; b += T) {
        uint32_t s = 0;
        if (before)
            for (uint32_t r = 0; r < c; ++r)
                s += __ldcg(cta_cnt + (size_t)r * MB + b);
        else
            for (uint32_t r = c + 1u; r < G; ++r)
                s += __ldcg(cta_cnt + (size_t)r * MB + b);
        const uint32_t total = (uint32_t)ld_relaxed_u64(&hdr->total[b]);
        tot[b] = total;
        run_base[b] = before ? s : total - cnt[b] - s;
        bin_tot[b] = fdc.div(total) + (fdc.mod(total) != 0u ? 1u : 0u); // chunks of port b
    }
    __syncthreads();
    const uint32_t R = block_exclusive_scan<T>(bin_tot, bin_base, B, scan_tmp);
    if (threadIdx.x == 0 && R > n_reserved)
        set_status(status, GF_OVERFLOW);
    // table [binBase | chunk ids] and descriptors, spread over the CTAs
    for (uint32_t r = c * (uint32_t)T + threadIdx.x; r < R; r += G * (uint32_t)T) {
        if (r >= fin.desc_cap || r >= n_reserved) {
            set_status(status, GF_OVERFLOW);
            continue;
        }
        uint32_t lo = 0, hi = B - 1u;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (bin_base[mid] <= r)
                lo = mid;
            else
                hi = mid - 1u;
        }
        const uint32_t k = r - bin_base[lo];
        const uint32_t chunk = __ldg(reserved + r);
        fin.table[B + r] = chunk;
        fin.descs[r].chunk_index = chunk;
        fin.descs[r].fill = min(capacity, tot[lo] - k * capacity);
        fin.descs[r].bin = lo;
    }
    if (c == 0) {
        for (uint32_t b = threadIdx.x; b < B; b += T) {
            fin.table[b] = bin_base[b];
            totals[b] = tot[b];
        }
        if (threadIdx.x == 0)
            *fin.num_out = R;
    }
    if (threadIdx.x == 0)
        misc[0] = ld_relaxed_u32(status);
    __syncthreads();
    if (misc[0] != 0u)
        return; // the batch failed: write nothing, the host discards it

    // ---------------- phase 2: rank, update, stage and write every tile ----------------
    for (uint32_t t = t_lo; t < t_hi; ++t) {
        uint64_t base = 0;
        const uint32_t count = tile_of(t, base);
        uint32_t bp[IPT];
        P p[IPT];
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            bp[r] = kNoBin16;
            if (i < count) {
                p[r] = acc.load(base + i);
                bp[r] = bins16[(size_t)t * Shape::kTile + i];
            }
        }
        warp_rank<Shape>(bp, warp_cnt, B);
        __syncthreads();
        warp_offsets<Shape>(warp_cnt, bin_tot, B);
        __syncthreads();
        const uint32_t n_valid = block_exclusive_scan<T>(bin_tot, bin_excl, B, scan_tmp);
#pragma unroll
        for (int r = 0; r < IPT; ++r) {
            const uint32_t b = bp_bin(bp[r]);
            if (b != kNoBin16) {
                const uint32_t q = bin_excl[b] + warp_cnt[(size_t)w * B + b] + bp_pos(bp[r]);
                const uint32_t res = update(b, p[r], seed_mixed);
                if (res != kUpdateSuccess)
                    set_status(status, res == kUpdateOverflow ? GF_OVERFLOW : GF_INVALID);
                stage[q] = p[r];
                stage_bin[q] = b;
            }
        }
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < n_valid; q += T) {
            const uint32_t b = stage_bin[q];
            const uint32_t j = run_base[b] + (q - bin_excl[b]);
            const uint32_t k = fdc.div(j);
            const uint32_t f = bin_base[b] + k;
            const uint32_t chunk = f < R && f < n_reserved ? __ldg(reserved + f) : kNoChunk;
            const uint64_t slot = (uint64_t)chunk * capacity + (j - k * capacity);
            if (chunk != kNoChunk && slot < pool_slots)
                acc.store(slot, stage[q]);
            else
                set_status(status, GF_OVERFLOW);
        }
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < B; b += T)
            run_base[b] += bin_tot[b];
        __syncthreads();
    }
    // the last CTA to finish runs the caller's post step over the published descriptors (every
    // other CTA's descriptors, output count and reads of its input are done before its arrival)
    if constexpr (Post::kActive) {
        if (threadIdx.x == 0) {
            __threadfence();
            misc[1] = atomicAdd(&hdr->finished, 1ull) + 1ull == (unsigned long long)G ? 1u : 0u;
        }
        __syncthreads();
        if (misc[1] != 0u) {
            __threadfence();
            post(fin, status);
        }
    }
}

// Host side: one cooperative launch over n_tiles tiles; the grid is as many CTAs as fit on the
// device at once (at most n_tiles and max_ctas). The scratch (any_coop_scratch_bytes) holds the
// header, zeroed here on the stream, the per-CTA rows and the bins.
// post: work of the last CTA after the whole batch (NoPost: none); zero_hdr false when an earlier
// launch on the stream has zeroed the header (sizeof(AnyCoopHdr) bytes at the scratch's start).
template <typename Shape, typename Access, typename Classify, typename Update, typename Post = NoPost>
cudaError_t launch_fused_any_coop(cudaStream_t stream, Access acc, Classify cls, Update upd, uint64_t seed_mixed,
                                  uint32_t capacity, uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles,
                                  uint32_t B, const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                                  void* scratch, uint64_t scratch_bytes, uint32_t max_ctas, uint32_t* status,
                                  InlineFinish fin, int sms, Post post = Post{}, bool zero_hdr = true)
{
    using P = typename Access::Payload;
    if (B == 0u || B > kAnyCoopMaxBins || fin.table == nullptr || n_tiles == 0u || scratch == nullptr ||
        (reinterpret_cast<uintptr_t>(scratch) & 15u) != 0u ||
        scratch_bytes < any_coop_scratch_bytes(n_tiles, Shape::kTile, max_ctas))
        return cudaErrorInvalidValue;
    auto kernel = fused_partition_any_coop_kernel<Shape, Access, Classify, Update, Post>;
    const size_t smem = any_coop_smem_bytes<Shape, P>(B);
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess)
        return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, Shape::kThreads, smem);
    if (err != cudaSuccess)
        return err;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    uint64_t g = (uint64_t)per_sm * (uint64_t)sms;
    g = g < n_tiles ? g : n_tiles;
    g = g < max_ctas ? g : max_ctas;
    auto* hdr = static_cast<AnyCoopHdr*>(scratch);
    auto* cta_cnt = reinterpret_cast<uint32_t*>(hdr + 1);
    auto* bins16 = reinterpret_cast<uint16_t*>(cta_cnt + (size_t)kAnyCoopMaxBins * max_ctas);
    if (zero_hdr) {
        err = cudaMemsetAsync(hdr, 0, sizeof(AnyCoopHdr), stream);
        if (err != cudaSuccess)
            return err;
    }
    FastDiv fd(capacity);
    void* args[] = {&acc,      &cls,      &upd,    &seed_mixed, &capacity, &fd,     &pool_slots,
                    &tiles,    &n_tiles,  &B,      &reserved,   &n_reserved, &totals, &hdr,
                    &cta_cnt,  &bins16,   &status, &fin,        &post};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3((uint32_t)g),
                                       dim3(Shape::kThreads), args, smem, stream);
}

} // namespace
} // namespace gf
