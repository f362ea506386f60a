// Persistent fused classify -> scan -> scatter for u32 keys and up to 64 dense ports, with
// bulk-copy (TMA engine) double buffering of the input tiles.
//
// Same contract and scratch layout as fused_partition_kernel (gf_partition.cuh): per tile a stable
// in-tile rank, a decoupled look-back per port over 64-bit (epoch | flag | value) descriptors,
// first-touch claims of output chunks from the caller's reservation, and a coalesced write-out.
// What differs is how the tile is processed:
//   * persistent CTAs take tiles from the launch counter in order; while a CTA processes tile t,
//     the bulk copy of its next tile into the other shared buffer is already in flight
//     (cp.async.bulk global -> shared, completion on an mbarrier; no multicast);
//   * thread i owns the 16 consecutive keys [16i, 16i + 16) of the tile; ranks come from per-thread
//     16-bit counters packed two per word ([rows][threads], bin b in row b % rows, half b / rows)
//     and one padded raking scan, so the order inside a port is (tile, bin, thread, item) = input
//     order;
//   * the staged tile is written out in 256-item segments spread evenly over the warps.
#pragma once

#include "gf_partition.cuh"

namespace gf {
namespace { // internal linkage: see gf_partition.cuh

GF_D uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

GF_D void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

GF_D void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

GF_D void proxy_async_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

GF_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared of `bytes` (multiple of 16, both addresses 16-byte aligned).
GF_D void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

GF_D bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0u;
}

template <int THREADS, int IPT>
struct TmaShape {
    static constexpr int kThreads = THREADS;
    static constexpr int kIpt = IPT;
    static constexpr int kWarps = THREADS / 32;
    static constexpr int kTile = THREADS * IPT;
    static constexpr int kLogThreads = THREADS == 256 ? 8 : (THREADS == 512 ? 9 : 7);
    static constexpr uint32_t kMaxBins = 64u;
    static constexpr uint32_t kSeg = 256u; // write-out segment
    // shared memory layout (32-bit words)
    static constexpr uint32_t kInbuf = 0;                                  // [2][TILE]
    static constexpr uint32_t kStage = kInbuf + 2u * kTile;                // [TILE]
    static constexpr uint32_t kCnt = kStage + kTile;                       // [THREADS * 33]
    static constexpr uint32_t kBStart = kCnt + THREADS * 33u;              // [65]
    static constexpr uint32_t kBTot = kBStart + 65u;                       // [64]
    static constexpr uint32_t kGP = kBTot + 64u;                           // [64]
    static constexpr uint32_t kLoBase = kGP + 64u;                         // [64]
    static constexpr uint32_t kHiBase = kLoBase + 64u;                     // [64]
    static constexpr uint32_t kCapLo = kHiBase + 64u;                      // [64]
    static constexpr uint32_t kSegStart = kCapLo + 64u;                    // [65]
    static constexpr uint32_t kLbFlag = kSegStart + 65u;                   // [THREADS]
    static constexpr uint32_t kLbVal = kLbFlag + THREADS;                  // [THREADS]
    static constexpr uint32_t kScanTmp = kLbVal + THREADS;                 // [W + 1]
    static constexpr uint32_t kMisc = kScanTmp + kWarps + 1u;              // [8]
    static constexpr uint32_t kMbar = (kMisc + 8u + 1u) & ~1u;             // 2 x u64, 8-byte aligned
    static constexpr uint32_t kWords = kMbar + 4u;
    static constexpr size_t kSmemBytes = sizeof(uint32_t) * kWords;
};

// Rotate the four 16-byte groups of a thread's 16 keys back into order: v[c] holds group
// (c + rot) & 3 (the lane-dependent rotation that makes the shared loads bank-conflict free).
GF_D void unrotate16(uint4 (&v)[4], uint32_t rot)
{
    if (rot & 1u) { // rotate by one group
        const uint4 t = v[3];
        v[3] = v[2];
        v[2] = v[1];
        v[1] = v[0];
        v[0] = t;
    }
    if (rot & 2u) { // rotate by two groups
        uint4 t = v[0];
        v[0] = v[2];
        v[2] = t;
        t = v[1];
        v[1] = v[3];
        v[3] = t;
    }
}

template <typename Shape, typename Classify>
__global__ void __launch_bounds__(Shape::kThreads, 2)
    fused_partition_tma_kernel(const uint32_t* __restrict__ in, uint32_t* out, Classify classify, uint32_t capacity,
                               FastDiv fdc, uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t B,
                               uint32_t rows_log2, const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                               unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl,
                               unsigned long long* desc, uint32_t* status)
{
    static_assert(Shape::kIpt == 16, "the TMA kernel reads 16 keys (four 16-byte groups) per thread");
    constexpr int T = Shape::kThreads, IPT = Shape::kIpt, W = Shape::kWarps;
    constexpr uint32_t TILE = Shape::kTile;
    extern __shared__ __align__(128) uint32_t sm[];
    uint32_t* inbuf = sm + Shape::kInbuf;
    uint32_t* stage = sm + Shape::kStage;
    uint32_t* cnt = sm + Shape::kCnt;
    uint32_t* bstart = sm + Shape::kBStart;
    uint32_t* btot = sm + Shape::kBTot;
    uint32_t* gP = sm + Shape::kGP;
    uint32_t* loBase = sm + Shape::kLoBase;
    uint32_t* hiBase = sm + Shape::kHiBase;
    uint32_t* capLo = sm + Shape::kCapLo;
    uint32_t* segStart = sm + Shape::kSegStart;
    uint32_t* lbFlag = sm + Shape::kLbFlag;
    uint32_t* lbVal = sm + Shape::kLbVal;
    uint32_t* scanTmp = sm + Shape::kScanTmp;
    uint32_t* misc = sm + Shape::kMisc; // 0 tile, 1 next tile, 2 epoch, 3 status, 4/5 bytes loaded per buffer
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + Shape::kMbar);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t rows = 1u << rows_log2, rmask = rows - 1u, stride = rows == 1u ? 1u : rows + 1u;

    // issue the bulk copy of tile `t` into buffer `buf` (thread 0 only); records the byte count
    auto issue = [&](uint32_t t, uint32_t buf) {
        uint32_t bytes = 0u;
        if (t < n_tiles) {
            const gf_tile tl = tiles[t];
            const uint64_t base = (uint64_t)tl.chunk_index * capacity + tl.tile_offset;
            const bool ok = tl.count != 0u && tl.count <= TILE && base + tl.count <= pool_slots &&
                            tl.tile_offset + tl.count <= capacity && (base & 3u) == 0u && (capacity & 3u) == 0u;
            if (ok) {
                bytes = ((tl.count + 3u) & ~3u) * 4u;
                proxy_async_fence();
                mbar_expect_tx(&mbar[buf], bytes);
                bulk_load(inbuf + buf * TILE, in + base, bytes, &mbar[buf]);
            } else {
                set_status(status, GF_INVALID);
            }
        }
        misc[4 + buf] = bytes;
    };

    // Static round-robin schedule under a cooperative launch: CTA c takes tiles c, c + G, c + 2G, ...
    // in order. Every CTA is resident, so every tile a look-back waits on is being processed (or
    // is the next tile of a CTA that is processing an earlier one) and no tile waits on a CTA
    // that has not started.
    if (tid == 0) {
        mbar_init(&mbar[0], 1u);
        mbar_init(&mbar[1], 1u);
        mbar_init_fence();
        misc[2] = next_epoch(ld_relaxed_u32(&ctl->epoch));
    }
    __syncthreads();
    uint32_t t = blockIdx.x;
    const uint32_t epoch = misc[2];
    if (tid == 0)
        issue(t, 0u);
    uint32_t cur = 0u, parity0 = 0u, parity1 = 0u;

    while (t < n_tiles) {
        if (tid == 0) {
            const uint32_t tn = t + gridDim.x;
            misc[1] = tn;
            issue(tn, cur ^ 1u);
        }
        // zero this tile's counters while the copy lands
        for (uint32_t i = tid; i < (uint32_t)T * stride; i += T)
            cnt[i] = 0u;
        __syncthreads();
        const uint32_t tn = misc[1];
        const gf_tile tile = tiles[t];
        const uint32_t bytes = misc[4 + cur];
        bool loaded = bytes != 0u;
        if (loaded) {
            const uint32_t par = cur == 0u ? parity0 : parity1;
            uint32_t polls = 0;
            while (!mbar_try_wait(&mbar[cur], par)) {
                if (++polls > kSpinLimit) {
                    set_status(status, GF_ERR_TIMEOUT);
                    loaded = false;
                    break;
                }
            }
            if (cur == 0u)
                parity0 ^= 1u;
            else
                parity1 ^= 1u;
        }
        const uint32_t n = loaded ? tile.count : 0u;

        // 1. classify my 16 keys (input order) and count them in my counter column
        uint4 v[4];
        const uint32_t rot = (lane >> 1) & 3u;
        const uint4* src = reinterpret_cast<const uint4*>(inbuf + cur * TILE + tid * IPT);
#pragma unroll
        for (int c = 0; c < 4; ++c)
            v[c] = src[(c + rot) & 3u];
        unrotate16(v, rot);
        uint32_t key[IPT];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            key[4 * c + 0] = v[c].x;
            key[4 * c + 1] = v[c].y;
            key[4 * c + 2] = v[c].z;
            key[4 * c + 3] = v[c].w;
        }
        uint32_t bp[IPT];
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            bp[k] = kNoBin16;
            if (tid * IPT + k < n) {
                const uint32_t b = classify(key[k]);
                if (b >= B) {
                    set_status(status, GF_INVALID);
                } else {
                    const uint32_t s = ((b & rmask) << Shape::kLogThreads) + tid;
                    const uint32_t a = (s >> rows_log2) * stride + (s & rmask);
                    const uint32_t sh = (b >> rows_log2) << 4;
                    const uint32_t old = cnt[a];
                    cnt[a] = old + (1u << sh);
                    bp[k] = b | (((old >> sh) & 0xFFFFu) << 16);
                }
            }
        }
        __syncthreads();

        // 2. padded raking scan: thread i owns scan entries [i*rows, (i+1)*rows)
        uint32_t sum = 0;
        for (uint32_t i = 0; i < rows; ++i)
            sum += cnt[tid * stride + i];
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (uint32_t)o)
                incl += x;
        }
        if (lane == 31u)
            scanTmp[warp] = incl;
        __syncthreads();
        if (tid == 0) {
            uint32_t run = 0;
            for (int i = 0; i < W; ++i) {
                const uint32_t c = scanTmp[i];
                scanTmp[i] = run;
                run += c;
            }
            scanTmp[W] = run;
        }
        __syncthreads();
        {
            uint32_t run = scanTmp[warp] + incl - sum;
            for (uint32_t i = 0; i < rows; ++i) {
                const uint32_t c = cnt[tid * stride + i];
                cnt[tid * stride + i] = run;
                run += c;
            }
        }
        const uint32_t total = scanTmp[W];
        const uint32_t totalLo = total & 0xFFFFu;
        const uint32_t nValid = totalLo + (total >> 16);
        __syncthreads();

        // 3. per-bin tile starts/totals, aggregate descriptor
        unsigned long long* myDesc = desc + (size_t)t * B;
        if (tid < B) {
            const uint32_t s = (tid & rmask) << Shape::kLogThreads;
            const uint32_t a = (s >> rows_log2) * stride + (s & rmask);
            const uint32_t h = tid >> rows_log2;
            bstart[tid] = ((cnt[a] >> (h << 4)) & 0xFFFFu) + (h ? totalLo : 0u);
        }
        if (tid == 0)
            bstart[B] = nValid;
        __syncthreads();
        if (tid < B) {
            btot[tid] = bstart[tid + 1] - bstart[tid];
            st_relaxed_u64(myDesc + tid, make_desc(epoch, t == 0 ? 2u : 1u, btot[tid]));
        }

        // 4. stage the tile in port order (tile-local positions only)
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const uint32_t b = bp_bin(bp[k]);
            if (b != kNoBin16) {
                const uint32_t s = ((b & rmask) << Shape::kLogThreads) + tid;
                const uint32_t a = (s >> rows_log2) * stride + (s & rmask);
                const uint32_t h = b >> rows_log2;
                const uint32_t q = ((cnt[a] >> (h << 4)) & 0xFFFFu) + (h ? totalLo : 0u) + bp_pos(bp[k]);
                stage[q] = key[k];
            }
        }

        // 5. look-back for the exclusive prefix of every port (gP), loBase used as done flags
        if (t != 0u)
            block_lookback<T>(desc, t, B, epoch, gP, loBase, lbFlag, lbVal, status);
        else if (tid < B)
            gP[tid] = 0u;
        __syncthreads();

        // 6. publish inclusive prefixes, claim this tile's output chunks, segment counts
        if (tid < B) {
            const uint32_t excl = gP[tid], tot = btot[tid];
            if (t != 0u)
                st_relaxed_u64(myDesc + tid, make_desc(epoch, 2u, excl + tot));
            if (t + 1u == n_tiles)
                totals[tid] = excl + tot;
            uint32_t lo = kNoChunk, hi = kNoChunk, cap = 0u;
            if (tot != 0u) {
                const uint32_t ka = fdc.div(excl), kb = fdc.div(excl + tot - 1u);
                cap = (ka + 1u) * capacity - excl;
                if (kb >= max_k) {
                    set_status(status, GF_OVERFLOW);
                } else {
                    lo = claim_chunk(port_chunks + (size_t)tid * max_k + ka, epoch, ctl, reserved, n_reserved, status);
                    if (kb != ka)
                        hi = claim_chunk(port_chunks + (size_t)tid * max_k + kb, epoch, ctl, reserved, n_reserved,
                                         status);
                }
                const uint32_t within = excl - ka * capacity;
                loBase[tid] = lo == kNoChunk ? kNoChunk : lo * capacity + within;
                hiBase[tid] = (kb == ka || hi == kNoChunk) ? kNoChunk : hi * capacity - cap;
            } else {
                loBase[tid] = kNoChunk;
                hiBase[tid] = kNoChunk;
            }
            capLo[tid] = cap;
        }
        if (warp == 0) { // segments of 256 items per port, exclusive scan over <= 64 ports
            const uint32_t b0 = 2u * lane, b1 = b0 + 1u;
            const uint32_t c0 = b0 < B ? (bstart[b0 + 1] - bstart[b0] + Shape::kSeg - 1u) / Shape::kSeg : 0u;
            const uint32_t c1 = b1 < B ? (bstart[b1 + 1] - bstart[b1] + Shape::kSeg - 1u) / Shape::kSeg : 0u;
            uint32_t inc = c0 + c1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, inc, o);
                if (lane >= (uint32_t)o)
                    inc += x;
            }
            const uint32_t ex = inc - c0 - c1;
            if (b0 < B)
                segStart[b0] = ex;
            if (b1 < B)
                segStart[b1] = ex + c0;
            if (lane == 31u)
                segStart[B] = inc; // bins >= B add nothing, so lane 31 holds the total
        }
        if (tid == 0)
            misc[3] = ld_relaxed_u32(status);
        __syncthreads();

        // 7. write-out: warps take 256-item segments round robin
        if (misc[3] == 0u) {
            const uint32_t nseg = segStart[B];
            for (uint32_t sg = warp; sg < nseg; sg += W) {
                uint32_t lo = 0, hi = B; // largest b with segStart[b] <= sg
                while (hi - lo > 1u) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (segStart[mid] <= sg)
                        lo = mid;
                    else
                        hi = mid;
                }
                const uint32_t b = lo;
                const uint32_t off = (sg - segStart[b]) * Shape::kSeg;
                const uint32_t nb = min(Shape::kSeg, btot[b] - off);
                const uint32_t lb = loBase[b], hb = hiBase[b], cap = capLo[b], from = bstart[b] + off;
                for (uint32_t i = lane; i < nb; i += 32u) {
                    const uint32_t j = off + i;
                    const uint32_t dst = j < cap ? lb + j : hb + j;
                    const bool ok = j < cap ? lb != kNoChunk : hb != kNoChunk;
                    if (ok && dst < pool_slots)
                        out[dst] = stage[from + i];
                }
            }
        }
        t = tn;
        cur ^= 1u;
    }
    fused_retire(ctl, epoch);
}

} // namespace
} // namespace gf
