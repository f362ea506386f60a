// Fused classify -> plan -> scatter of one whole batch in a single cooperative launch, for u32
// keys and up to 64 dense ports.
//
// Same contract and results as fused_partition_kernel (gf_partition.cuh): per-port totals, the
// exact plan, and every port's keys in input order. What differs is how a tile learns where its
// keys go. At B200 rates (tens of tiles per microsecond) a decoupled look-back makes every tile
// wait for, and sum, the aggregates of the many tiles still in flight; this kernel takes one grid
// barrier instead:
//   phase 1  every CTA counts the keys of its contiguous range of tiles: bulk copies (TMA engine)
//            keep three tiles in flight per CTA, threads count with packed 16-bit counters;
//   barrier  cooperative launch (all CTAs resident), bounded wait;
//   plan     every CTA reads all CTAs' per-port totals and derives its own per-port base and the
//            reference's dense plan, binBase[b] = sum_{b'<b} ceil(total_b' / C)
//            (graph/DenseBinTable.hpp:39-91); port b's k-th output chunk is reserved[binBase[b] + k],
//            so the chunk table equals the host plan's; the chunk ids this CTA will write to are
//            fetched once into shared memory;
//   phase 2  every CTA walks its tiles again, last tile first (the last tiles it counted are the ones
//            still in L2). Per tile: a bulk copy two tiles ahead, a stable rank from per-thread packed
//            counters and one padded raking scan (cost independent of the port distribution),
//            staging in port order (each key with its output slot; with capacity >= 4096 a port's
//            run of one tile touches at most two output chunks), and a write-out in which every
//            thread stores stage positions tid, tid + 256, ... (coalesced along each run).
// Requirements (checked by the dispatcher): B <= 64, tiles of at most 4096 keys, capacity % 4 == 0
// and >= 4096, at most 2^32 pool slots, key columns 16-byte aligned, scratch for 64 words per CTA.
#pragma once

#include "gf_partition.cuh"

namespace gf {
namespace { // internal linkage: see gf_partition.cuh

GF_D uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

GF_D void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

GF_D void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

GF_D void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

GF_D void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

GF_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

GF_D bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0u;
}

// Bounded wait for the phase of `parity` to complete; gives up with GF_ERR_TIMEOUT.
GF_D void mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* status)
{
    uint32_t polls = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++polls >= kSpinLimit) {
            set_status(status, GF_ERR_TIMEOUT);
            return;
        }
    }
}

// 1-D bulk copy global -> shared of `bytes` (multiple of 16, both addresses 16-byte aligned),
// completing on `bar`. No multicast.
GF_D void bulk_load(void* sdst, const void* gsrc, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(sdst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

GF_D uint32_t ld_acquire_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Built-in key classifiers of the specialised kernel (a result >= bins is invalid).
struct MaskClassify { // key mod B for B a power of two
    uint32_t mask;
    GF_D uint32_t operator()(uint32_t k) const { return k & mask; }
};
struct ModClassify { // key mod B
    FastDiv fd;
    GF_D uint32_t operator()(uint32_t k) const { return fd.mod(k); }
};
struct AnyKeyClassify { // every other built-in rule
    KeyClassifier c;
    GF_D uint32_t operator()(uint32_t k) const { return c((uint64_t)k); }
};

// 256 threads; LANES counter rows with two ports per row (up to 2 * LANES ports).
template <int LANES>
struct CoopShape {
    static constexpr int kThreads = 256;
    static constexpr int kWarps = kThreads / 32;
    // Phase 2: thread t owns the 17 consecutive keys [17 t, 17 t + 17). An odd count makes the 32
    // stage stores of a warp that all belong to one port run land in 32 different banks.
    static constexpr int kIpt = 17;
    static constexpr uint32_t kMaxCount = 4096u; // keys per tile
    static constexpr uint32_t kInWords = (uint32_t)kThreads * kIpt;
    static constexpr uint32_t kLanes = LANES;
    static constexpr uint32_t kLaneShift = LANES == 2 ? 1u : (LANES == 8 ? 3u : 5u);
    static constexpr uint32_t kMaxBins = 2u * LANES;
    static constexpr uint32_t kBM = 64u; // per-port arrays are 64 wide whatever LANES is
    static constexpr uint32_t kMinCapacity = kMaxCount; // one tile's run of a port touches <= 2 chunks
    static constexpr uint32_t kSeg = LANES + 1u;                           // raking segment (padded)
    static constexpr uint32_t kIdCache = 512u; // chunk ids of this CTA's output held in shared memory
    // shared memory (32-bit words). Phase 2 stages a tile in its own input buffer (its keys are in
    // registers by then); phase 1's three-tile ring is in[0], in[1] and the slot array.
    static constexpr uint32_t kIn = 0;                              // [2][kInWords]
    static constexpr uint32_t kStage = kIn + 2u * kInWords;         // [kMaxCount] output slot per stage position
    static constexpr uint32_t kRun = kStage + kMaxCount;            // [65] stage start of each port's run
    // [64] x {stage position where the second chunk starts, slot - stage position in the first
    // chunk, the same in the second chunk, unused}: one 16-byte load per staged key
    static constexpr uint32_t kPort = (kRun + kBM + 4u + 3u) & ~3u;
    static constexpr uint32_t kOff = kPort + 4u * kBM;              // [64] running port position
    static constexpr uint32_t kCnt = kOff + kBM;                    // [kSeg][kThreads]
    static constexpr uint32_t kBase = kCnt + kSeg * kThreads;       // [64] this CTA's first port position
    static constexpr uint32_t kTotal = kBase + kBM;                 // [64] batch totals
    static constexpr uint32_t kBinBase = kTotal + kBM;              // [64] dense plan
    static constexpr uint32_t kOwn = kBinBase + kBM;                // [64] this CTA's totals
    static constexpr uint32_t kKfirst = kOwn + kBM;                 // [64] first output chunk of the range
    static constexpr uint32_t kAcc = kKfirst + kBM;                 // [64] phase-1 flushed counts
    static constexpr uint32_t kIdOff = kAcc + kBM;                  // [65] id cache offsets
    static constexpr uint32_t kIds = kIdOff + kBM + 4u;             // [kIdCache]
    static constexpr uint32_t kScan = kIds + kIdCache;              // [W]
    static constexpr uint32_t kTiles = kScan + kWarps;              // [6][4] buffered tile descriptors
    static constexpr uint32_t kMisc = kTiles + 24u;                 // [8]
    static constexpr uint32_t kMbar = (kMisc + 8u + 1u) & ~1u;      // [3] x u64
    static constexpr uint32_t kWords = kMbar + 6u;
    static constexpr size_t kSmemBytes = sizeof(uint32_t) * kWords;
    GF_D static uint32_t ring(uint32_t buf) { return buf == 0u ? kIn : buf == 1u ? kIn + kInWords : kStage; }
};

// Grid-wide barrier of a cooperative launch on a counter reset before the launch. Bounded: a wait
// that gives up sets GF_ERR_TIMEOUT and returns.
GF_D void coop_grid_barrier(uint32_t* counter, uint32_t* status)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(counter, 1u);
        uint32_t polls = 0;
        while (ld_acquire_u32(counter) < gridDim.x) {
            if (++polls >= kSpinLimit) {
                set_status(status, GF_ERR_TIMEOUT);
                break;
            }
            __nanosleep(polls < 64u ? 32u : 128u);
        }
        __threadfence();
    }
    __syncthreads();
}

// Thread 0: fetch tile `t` into the shared buffer at word offset `dst` (bulk copy completing on
// `bar`, or a plain arrival when the tile cannot be bulk copied) and describe it in d[0..3]:
// chunk, offset, count (0 for an invalid tile), flags (1 = valid, 2 = in shared memory).
GF_D void coop_fetch(const gf_tile* tiles, uint32_t t, const uint32_t* in, uint32_t capacity, uint64_t pool_slots,
                     uint32_t max_count, uint32_t* sm, uint32_t dst, uint64_t* bar, uint32_t* d, uint32_t* status)
{
    const gf_tile tile = tiles[t];
    const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
    const bool ok =
        tile.count <= max_count && base + tile.count <= pool_slots && tile.tile_offset + tile.count <= capacity;
    if (!ok)
        set_status(status, GF_INVALID);
    const uint32_t words = (tile.count + 3u) & ~3u;
    const bool bulk = ok && (base & 3u) == 0u && words != 0u && base + words <= pool_slots;
    d[0] = tile.chunk_index;
    d[1] = tile.tile_offset;
    d[2] = ok ? tile.count : 0u;
    d[3] = (ok ? 1u : 0u) | (bulk ? 2u : 0u);
    if (bulk) {
        mbar_expect_tx(bar, words * 4u);
        bulk_load(sm + dst, in + base, words * 4u, bar);
    } else {
        mbar_arrive(bar); // the phase completes; the keys are read from global memory
    }
}

template <typename S, typename Classify>
__global__ void __launch_bounds__(S::kThreads, 2)
    fused_partition_coop_kernel(const uint32_t* __restrict__ in, uint32_t* out, Classify cls, uint32_t capacity,
                                FastDiv fdc, uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t B,
                                const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                                unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl, uint32_t* cta_tot,
                                uint32_t* status)
{
    constexpr int T = S::kThreads, IPT = S::kIpt, W = S::kWarps;
    constexpr uint32_t BM = S::kBM, L = S::kLanes, SEG = S::kSeg;
    extern __shared__ __align__(128) uint32_t sm[];
    uint32_t* cnt = sm + S::kCnt;
    uint32_t* cbase = sm + S::kBase;
    uint32_t* total = sm + S::kTotal;
    uint32_t* bin_base = sm + S::kBinBase;
    uint32_t* run_at = sm + S::kRun;
    uint4* port4 = reinterpret_cast<uint4*>(sm + S::kPort);
    uint32_t* off = sm + S::kOff;
    uint32_t* oslot = sm + S::kStage;
    uint32_t* own = sm + S::kOwn;
    uint32_t* kfirst = sm + S::kKfirst;
    uint32_t* acc = sm + S::kAcc;
    uint32_t* idoff = sm + S::kIdOff;
    uint32_t* ids = sm + S::kIds;
    uint32_t* scan = sm + S::kScan;
    uint32_t* tdesc = sm + S::kTiles;
    uint32_t* misc = sm + S::kMisc;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + S::kMbar);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    const uint32_t G = gridDim.x, c = blockIdx.x;

    // this CTA's tiles: [t_lo, t_hi) of an even split
    const uint32_t t_lo = (uint32_t)((uint64_t)n_tiles * c / G);
    const uint32_t t_hi = (uint32_t)((uint64_t)n_tiles * (c + 1u) / G);
    const uint32_t n_mine = t_hi - t_lo;
    if (tid == 0) {
        misc[0] = next_epoch(ld_relaxed_u32(&ctl->epoch));
#pragma unroll
        for (int i = 0; i < 3; ++i)
            mbar_init(&mbar[i], 1u);
        mbar_init_fence();
    }
    for (uint32_t i = tid; i < SEG * T; i += T)
        cnt[i] = 0u;
    if (tid < BM)
        acc[tid] = 0u;
    __syncthreads();
    const uint32_t epoch = misc[0];

    // ---------------- phase 1: per-port counts of this CTA's tiles (forward, three in flight) ----------------
    if (tid == 0)
        for (uint32_t q = 0; q < 3u && q < n_mine; ++q)
            coop_fetch(tiles, t_lo + q, in, capacity, pool_slots, S::kMaxCount, sm, S::ring(q), &mbar[q],
                       tdesc + 4u * q, status);
    bool bad = false;
    auto count_key = [&](uint32_t key) {
        const uint32_t b = cls(key);
        if (b < B) // own column: no contention; a reduction, so consecutive keys do not wait on each other
            atomicAdd(cnt + (b & (L - 1u)) * T + tid, 1u << ((b >> S::kLaneShift) << 4));
        else
            bad = true;
    };
    // adds the packed counters into acc[] and clears them (a thread counts at most 16 keys per tile,
    // so 2048 tiles between flushes keep every 16-bit counter below 2^15)
    auto flush = [&]() {
        for (uint32_t r = w; r < L; r += W) {
            uint32_t lo = 0, hi = 0;
            for (uint32_t i = lane; i < (uint32_t)T; i += 32u) {
                const uint32_t x = cnt[r * T + i];
                cnt[r * T + i] = 0u;
                lo += x & 0xFFFFu;
                hi += x >> 16;
            }
            lo = __reduce_add_sync(0xFFFFFFFFu, lo);
            hi = __reduce_add_sync(0xFFFFFFFFu, hi);
            if (lane == 0) {
                acc[r] += lo;
                acc[r + L] += hi;
            }
        }
        __syncthreads();
    };
    for (uint32_t q = 0; q < n_mine; ++q) {
        const uint32_t buf = q % 3u;
        const uint32_t* d = tdesc + 4u * buf;
        mbar_wait(&mbar[buf], (q / 3u) & 1u, status);
        const uint32_t count = d[2], flags = d[3];
        if (flags & 2u) {
            const uint4* v = reinterpret_cast<const uint4*>(sm + S::ring(buf));
#pragma unroll
            for (uint32_t j = 0; j < S::kMaxCount / 4u / (uint32_t)T; ++j) {
                const uint32_t vi = tid + j * (uint32_t)T;
                if (vi * 4u < count) {
                    const uint4 x = v[vi];
                    count_key(x.x);
                    if (vi * 4u + 1u < count)
                        count_key(x.y);
                    if (vi * 4u + 2u < count)
                        count_key(x.z);
                    if (vi * 4u + 3u < count)
                        count_key(x.w);
                }
            }
        } else if (flags & 1u) {
            const uint64_t base = (uint64_t)d[0] * capacity + d[1];
            for (uint32_t i = tid; i < count; i += T)
                count_key(__ldg(in + base + i));
        }
        fence_proxy_async_smem(); // this buffer's reads come before the next bulk copy into it
        __syncthreads();
        if (tid == 0 && q + 3u < n_mine)
            coop_fetch(tiles, t_lo + q + 3u, in, capacity, pool_slots, S::kMaxCount, sm, S::ring(buf), &mbar[buf],
                       tdesc + 4u * buf, status);
        if ((q & 2047u) == 2047u)
            flush();
    }
    if (bad)
        set_status(status, GF_INVALID);
    flush();
    if (tid < BM) {
        const uint32_t v = tid < B ? acc[tid] : 0u;
        own[tid] = v;
        cta_tot[(size_t)c * BM + tid] = v;
    }
    // phase 2 walks the tiles last to first through in[0] and in[1]; its first two tiles are
    // fetched across the barrier. Uses of each buffer so far set the mbarrier parities.
    const uint32_t use0 = (n_mine + 2u) / 3u, use1 = (n_mine + 1u) / 3u;
    if (tid == 0)
        for (uint32_t k = 0; k < 2u && k < n_mine; ++k)
            coop_fetch(tiles, t_hi - 1u - k, in, capacity, pool_slots, S::kMaxCount, sm, S::ring(k), &mbar[k],
                       tdesc + 16u + 4u * k, status);

    coop_grid_barrier(&ctl->done, status);

    // ---------------- plan ----------------
    {
        // thread tid covers port b = tid % 64 of CTAs c' = tid / 64, + 4, + 8, ...
        const uint32_t b = tid % BM;
        constexpr uint32_t kStride = (uint32_t)T / BM;
        uint32_t below = 0, all = 0;
        for (uint32_t c0 = tid / BM; c0 < G; c0 += kStride * 8u) {
            uint32_t v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const uint32_t cc = c0 + (uint32_t)u * kStride;
                v[u] = cc < G ? ld_relaxed_u32(cta_tot + (size_t)cc * BM + b) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const uint32_t cc = c0 + (uint32_t)u * kStride;
                all += v[u];
                below += cc < c ? v[u] : 0u;
            }
        }
        uint32_t* red = sm + S::kStage; // stage buffer 0 is unused until phase 2
        red[tid] = all;
        red[T + tid] = below;
        __syncthreads();
        if (tid < BM) {
            uint32_t a = 0, bl = 0;
#pragma unroll
            for (uint32_t j = 0; j < kStride; ++j) {
                a += red[j * BM + tid];
                bl += red[T + j * BM + tid];
            }
            total[tid] = tid < B ? a : 0u;
            cbase[tid] = tid < B ? bl : 0u;
        }
        __syncthreads();
        if (w == 0) {
            // binBase = exclusive scan of ceil(total / C); first chunk and chunk count of this CTA's
            // range per port (two ports per lane)
            const uint32_t b0 = 2u * lane, b1 = b0 + 1u;
            uint32_t n0 = 0, n1 = 0, m0 = 0, m1 = 0;
            if (b0 < B)
                n0 = fdc.div(total[b0]) + (fdc.mod(total[b0]) != 0u ? 1u : 0u);
            if (b1 < B)
                n1 = fdc.div(total[b1]) + (fdc.mod(total[b1]) != 0u ? 1u : 0u);
            const uint32_t kf0 = fdc.div(cbase[b0]), kf1 = fdc.div(cbase[b1]);
            if (own[b0] != 0u)
                m0 = fdc.div(cbase[b0] + own[b0] - 1u) - kf0 + 1u;
            if (own[b1] != 0u)
                m1 = fdc.div(cbase[b1] + own[b1] - 1u) - kf1 + 1u;
            kfirst[b0] = kf0;
            kfirst[b1] = kf1;
            uint32_t incl = n0 + n1, mincl = m0 + m1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                const uint32_t z = __shfl_up_sync(0xFFFFFFFFu, mincl, o);
                if ((int)lane >= o) {
                    incl += y;
                    mincl += z;
                }
            }
            const uint32_t ex = incl - n0 - n1, mex = mincl - m0 - m1;
            bin_base[b0] = ex;
            bin_base[b1] = ex + n0;
            idoff[b0] = mex;
            idoff[b1] = mex + m0;
            if (lane == 31) {
                idoff[BM] = mincl;
                misc[1] = incl; // R = chunks of the plan
                if (incl > n_reserved)
                    set_status(status, GF_OVERFLOW);
            }
        }
        __syncthreads();
        const uint32_t R = misc[1];
        // chunk ids of this CTA's output runs, once
        const uint32_t n_ids = idoff[BM] < S::kIdCache ? idoff[BM] : S::kIdCache;
        for (uint32_t i = tid; i < n_ids; i += T) {
            uint32_t lo = 0, hi = BM - 1u; // the last port whose run starts at or before i
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1u) >> 1;
                if (idoff[mid] <= i)
                    lo = mid;
                else
                    hi = mid - 1u;
            }
            const uint32_t f = bin_base[lo] + kfirst[lo] + (i - idoff[lo]);
            ids[i] = f < R && f < n_reserved ? __ldg(reserved + f) : kNoChunk;
        }
        // port b's chunk list, written by CTA b % G; batch totals and the epoch by CTA 0
        for (uint32_t pb = c; pb < B; pb += G) {
            const uint32_t nck = fdc.div(total[pb]) + (fdc.mod(total[pb]) != 0u ? 1u : 0u);
            if (nck > max_k) {
                if (tid == 0)
                    set_status(status, GF_OVERFLOW);
                continue;
            }
            for (uint32_t k = tid; k < nck; k += T) {
                const uint32_t f = bin_base[pb] + k;
                const uint32_t chunk = f < R && f < n_reserved ? __ldg(reserved + f) : kNoChunk;
                port_chunks[(size_t)pb * max_k + k] = ((unsigned long long)epoch << 32) | chunk;
            }
        }
        if (c == 0) {
            for (uint32_t b2 = tid; b2 < B; b2 += T)
                totals[b2] = total[b2];
            if (tid == 0)
                atomicExch(&ctl->epoch, epoch); // every CTA read the old epoch before the barrier
        }
        if (tid == 0)
            misc[2] = ld_relaxed_u32(status);
        __syncthreads();
    }
    const bool failed = misc[2] != 0u;
    const uint32_t R = misc[1];

    // chunk id of port b's k-th output chunk (k inside this CTA's range of the port)
    auto chunk_of = [&](uint32_t b, uint32_t k) -> uint32_t {
        const uint32_t rel = k - kfirst[b];
        if (rel < idoff[b + 1u] - idoff[b] && idoff[b] + rel < S::kIdCache)
            return ids[idoff[b] + rel];
        const uint32_t f = bin_base[b] + k;
        return f < R && f < n_reserved ? __ldg(reserved + f) : kNoChunk;
    };

    // running port positions: the end of this CTA's range (its tiles are walked last to first)
    if (tid < BM)
        off[tid] = cbase[tid] + own[tid];
    __syncthreads();

    // ---------------- phase 2: rank, stage, write (tiles last to first) ----------------
    for (uint32_t k = 0; k < n_mine; ++k) {
        const uint32_t buf = k & 1u;
        const uint32_t* d = tdesc + 16u + 4u * buf;
        uint32_t* tin = sm + S::ring(buf);
        uint32_t* stage = tin; // the keys are in registers once counted
        mbar_wait(&mbar[buf], ((buf == 0u ? use0 : use1) + (k >> 1)) & 1u, status);
        const uint32_t count = d[2], flags = d[3];
        uint32_t key[IPT];
        if (flags & 2u) {
#pragma unroll
            for (int i = 0; i < IPT; ++i)
                key[i] = tin[tid * IPT + (uint32_t)i];
        } else {
            const uint64_t base = (uint64_t)d[0] * capacity + d[1];
#pragma unroll
            for (int i = 0; i < IPT; ++i) {
                const uint32_t it = tid * IPT + (uint32_t)i;
                key[i] = it < count ? __ldg(in + base + it) : 0u;
            }
        }
        // count: local rank among this thread's earlier keys of the same port
        uint32_t bp[IPT];
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const uint32_t it = tid * IPT + (uint32_t)i;
            uint32_t b = kNoBin16, lr = 0;
            if (it < count) {
                b = cls(key[i]);
                if (b >= B)
                    b = kNoBin16; // reported by phase 1
            }
            if (b != kNoBin16) {
                const uint32_t sh = (b >> S::kLaneShift) << 4;
                uint32_t* ctr = cnt + (b & (L - 1u)) * T + tid;
                const uint32_t old = *ctr;
                *ctr = old + (1u << sh);
                lr = (old >> sh) & 0xFFFFu;
            }
            bp[i] = b | (lr << 16);
        }
        __syncthreads();

        // raking scan over the (lane, thread) counters, padded segments of SEG words
        uint32_t* seg = cnt + tid * SEG;
        uint32_t sum = 0;
#pragma unroll
        for (uint32_t i = 0; i < SEG; ++i)
            sum += seg[i];
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if ((int)lane >= o)
                incl += y;
        }
        if (lane == 31u)
            scan[w] = incl;
        __syncthreads();
        uint32_t wpre = 0, gtot = 0;
#pragma unroll
        for (int i = 0; i < W; ++i) {
            const uint32_t x = scan[i];
            wpre += (uint32_t)i < w ? x : 0u;
            gtot += x;
        }
        uint32_t run = wpre + incl - sum + ((gtot & 0xFFFFu) << 16); // high ports follow all low ports
#pragma unroll
        for (uint32_t i = 0; i < SEG; ++i) {
            const uint32_t x = seg[i];
            seg[i] = run;
            run += x;
        }
        __syncthreads();

        // per port (one thread each): its run's stage start, the stage position where its second
        // output chunk starts, and slot - stage position for each of the two chunks
        if (tid < BM) {
            const uint32_t b = tid;
            uint32_t s0 = count, s1 = count;
            if (b < B)
                s0 = (cnt[(b & (L - 1u)) * T] >> ((b >> S::kLaneShift) << 4)) & 0xFFFFu;
            if (b + 1u < B)
                s1 = (cnt[((b + 1u) & (L - 1u)) * T] >> (((b + 1u) >> S::kLaneShift) << 4)) & 0xFFFFu;
            const uint32_t len = b < B ? s1 - s0 : 0u;
            const uint32_t j0 = off[b] - len;
            off[b] = j0;
            run_at[b] = s0;
            uint32_t sp = s0 + len, sa = kNoChunk, sb = kNoChunk;
            if (len != 0u) {
                const uint32_t k0 = fdc.div(j0);
                const uint32_t room = (k0 + 1u) * capacity - j0; // slots left in the first chunk
                // a chunk id outside the pool writes nothing and fails the batch
                auto in_pool = [&](uint32_t ch) {
                    const bool okc = ch != kNoChunk && ((uint64_t)ch + 1u) * capacity <= pool_slots;
                    if (!okc && ch != kNoChunk)
                        set_status(status, GF_OVERFLOW);
                    return okc;
                };
                const uint32_t ca = chunk_of(b, k0);
                if (in_pool(ca))
                    sa = ca * capacity + (j0 - k0 * capacity) - s0;
                if (len > room) {
                    sp = s0 + room;
                    const uint32_t cb = chunk_of(b, k0 + 1u);
                    if (in_pool(cb))
                        sb = cb * capacity - sp;
                }
            }
            port4[b] = make_uint4(sp, sa, sb, 0u);
        }
        __syncthreads();

        // stage in port order (the stage position is the rank), each key with its output slot
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const uint32_t b = bp[i] & 0xFFFFu;
            if (b != kNoBin16) {
                const uint32_t word = cnt[(b & (L - 1u)) * T + tid];
                const uint32_t pos = ((word >> ((b >> S::kLaneShift) << 4)) & 0xFFFFu) + (bp[i] >> 16);
                const uint4 pp = port4[b];
                const uint32_t base = pos < pp.x ? pp.y : pp.z;
                stage[pos] = key[i];
                oslot[pos] = base == kNoChunk ? kNoChunk : base + pos;
            }
        }
        __syncthreads();

        // this thread's counter column is reset for the next tile (no other thread reads it now)
#pragma unroll
        for (uint32_t r = 0; r < SEG; ++r)
            cnt[r * T + tid] = 0u;

        // write-out: consecutive threads take consecutive stage positions (coalesced along each run)
        if (!failed) {
#pragma unroll 4
            for (uint32_t q = tid; q < count; q += T) {
                const uint32_t sl = oslot[q];
                if (sl != kNoChunk)
                    out[sl] = stage[q];
            }
        }
        fence_proxy_async_smem(); // this buffer's reads come before the next bulk copy into it
        __syncthreads();
        if (tid == 0 && k + 2u < n_mine)
            coop_fetch(tiles, t_hi - 1u - (k + 2u), in, capacity, pool_slots, S::kMaxCount, sm, S::ring(buf),
                       &mbar[buf], tdesc + 16u + 4u * buf, status);
    }
}

// Host side: one cooperative launch of the kernel with classifier `cls`; the grid is as many CTAs
// as fit on the device at once, capped by the tiles and by the scratch (64 words per CTA after the
// control block, whose reset words the caller zeroed on the stream).
template <typename S, typename Cls>
cudaError_t launch_fused_coop(cudaStream_t stream, Cls cls, const uint32_t* in, uint32_t* out, uint32_t capacity,
                              uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t bins,
                              const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                              unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl, uint64_t scratch_bytes,
                              uint32_t* status, int sms)
{
    auto kernel = fused_partition_coop_kernel<S, Cls>;
    cudaError_t err = cudaSuccess;
    if (S::kSmemBytes > 48u * 1024u) {
        err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmemBytes);
        if (err != cudaSuccess)
            return err;
    }
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, S::kThreads, S::kSmemBytes);
    if (err != cudaSuccess)
        return err;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    uint64_t g = (uint64_t)per_sm * (uint64_t)sms;
    g = g < n_tiles ? g : n_tiles;
    const uint64_t cap_ctas = (scratch_bytes - sizeof(FusedCtl)) / 256u;
    g = g < cap_ctas ? g : cap_ctas;
    if (g == 0u)
        return cudaErrorInvalidConfiguration;
    uint32_t* cta_tot = reinterpret_cast<uint32_t*>(ctl + 1);
    FastDiv fd(capacity);
    void* args[] = {&in,       &out,        &cls,    &capacity, &fd,          &pool_slots,  &tiles,
                    &n_tiles,  &bins,       &reserved, &n_reserved, &totals, &port_chunks, &max_k,
                    &ctl,      &cta_tot,    &status};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3((uint32_t)g), dim3(S::kThreads),
                                       args, S::kSmemBytes, stream);
}

} // namespace
} // namespace gf
