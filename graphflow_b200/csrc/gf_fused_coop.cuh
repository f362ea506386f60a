// Fused classify -> plan -> scatter of one whole batch in a single cooperative launch, for u32
// keys and up to 64 dense ports.
//
// Same contract and results as fused_partition_kernel (gf_partition.cuh): per-port totals, the
// exact plan, and every port's keys in input order. What differs is how a tile learns where its
// keys go. At B200 rates (tens of tiles per microsecond) a decoupled look-back makes every tile
// wait for, and sum, the aggregates of the many tiles still in flight; this kernel takes one grid
// barrier instead:
//   phase 1  every CTA counts the keys of its contiguous range of tiles: bulk copies (TMA engine)
//            keep the next tile in flight while threads count with packed 16-bit counters; the
//            CTA's per-port totals go to its row of the scratch and are added to the batch totals;
//   barrier  cooperative launch (all CTAs resident), bounded wait;
//   plan     every CTA derives its own per-port base (the sum of the rows before it, or the batch
//            total minus the rows after it, whichever is fewer rows) and the reference's dense
//            plan, binBase[b] = sum_{b'<b} ceil(total_b' / C) (graph/DenseBinTable.hpp:39-91); port
//            b's k-th output chunk is reserved[binBase[b] + k], so the chunk table equals the host
//            plan's; the chunk ids this CTA will write to are fetched once into shared memory;
//   phase 2  every CTA walks its tiles again, last tile first (the last tiles it counted are the ones
//            still in L2). Per tile: a stable rank from per-thread 16-bit counters (thread t owns 33
//            consecutive keys; shared-memory atomics return the local rank) and one padded raking
//            scan with 128-bit accesses; staging in port order in the tile's own buffer; warp 0 cuts
//            each port's run at its output-chunk boundary (at most two pieces) and marks where each
//            piece starts in a bitmap of stage positions; in the write-out warp w copies stage
//            positions [1024 w, 1024 w + 1024) in order, each lane finding its piece by a popcount
//            of the bitmap, so every store of a warp is a coalesced run of slots.
// Requirements (checked by the dispatcher): B <= 64, tiles of at most 4096 keys, capacity % 4 == 0
// and >= 4096, at most 2^32 pool slots, key columns 16-byte aligned, scratch for the control block
// and 4 * B_max bytes per CTA.
#pragma once

#include "gf_partition.cuh"

#include <type_traits>

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

GF_D unsigned long long ld_acquire_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Built-in key classifiers of the specialised kernel (a result >= bins is invalid).
struct MaskClassify { // key mod B for B a power of two
    static constexpr bool kAlwaysValid = true;
    uint32_t mask;
    GF_D uint32_t operator()(uint32_t k) const { return k & mask; }
};
struct ModClassify { // key mod B
    static constexpr bool kAlwaysValid = true;
    FastDiv fd;
    GF_D uint32_t operator()(uint32_t k) const { return fd.mod(k); }
};
struct AnyKeyClassify { // every other built-in rule
    KeyClassifier c;
    GF_D uint32_t operator()(uint32_t k) const { return c((uint64_t)k); }
};

// True for classifiers whose result is below the port count for every key.
template <typename C>
constexpr bool always_valid()
{
    if constexpr (requires { C::kAlwaysValid; })
        return C::kAlwaysValid;
    else
        return false;
}

// Control block of the cooperative kernel, right after the FusedCtl in the scratch; the launcher
// zeroes it on the stream before every launch. The per-CTA port totals follow it. The scratch may
// later serve the per-tile look-back kernel, which reads the same bytes as 64-bit descriptors
// whose bits 33..32 are a publication flag (gf_partition.cuh); everything this kernel leaves
// there reads as "not published": the control block holds 64-bit words below 2^32 and the per-CTA
// rows hold counts times four.
struct CoopHdr {
    unsigned long long total[64]; // batch per-port totals: atomic sums of the CTAs' counts
    unsigned long long done;      // grid-barrier arrivals
    unsigned long long pad[7];    // the per-CTA rows behind it start 64-byte aligned (128-bit loads)
};
static_assert(sizeof(CoopHdr) % 64u == 0u && sizeof(FusedCtl) % 64u == 0u, "row alignment");
constexpr uint32_t kCoopHdrResetBytes = sizeof(CoopHdr);

// 128 threads; LANES counter rows with two 16-bit port counters per word (up to 2 * LANES ports).
template <int LANES>
struct CoopShape {
    static constexpr int kThreads = 128;
    static constexpr int kWarps = kThreads / 32;
    // Phase 2: thread t owns the 33 consecutive keys [33 t, 33 t + 33). An odd count makes the key
    // loads of a warp, and the stage stores of a warp whose keys all belong to one port run, land
    // in 32 different banks.
    static constexpr int kIpt = 33;
    static constexpr uint32_t kMaxCount = 4096u; // keys per tile
    static constexpr uint32_t kInWords = (uint32_t)kThreads * kIpt;
    static constexpr uint32_t kLanes = LANES;
    static constexpr uint32_t kLaneShift = LANES == 2 ? 1u : (LANES == 8 ? 3u : 5u);
    static constexpr uint32_t kMaxBins = 2u * LANES;
    static constexpr uint32_t kBM = 64u; // per-port arrays are 64 wide whatever LANES is
    static constexpr uint32_t kMinCapacity = kMaxCount; // one tile's run of a port touches <= 2 chunks
    // Raking segment: a multiple of 4 words so that it is read and written with 128-bit accesses;
    // thread r's segment starts at word r * kSeg, which puts the eight threads of each quarter warp
    // on eight disjoint groups of four banks.
    static constexpr uint32_t kSeg = LANES == 2 ? 4u : LANES + 4u;
    static constexpr uint32_t kMaxPieces = 2u * kMaxBins; // a port's run of one tile is cut at most once
    static constexpr uint32_t kBmWords = kMaxCount / 32u;  // one bit per stage position
    // shared memory (32-bit words)
    static constexpr uint32_t kIn = 0;                              // [2][kInWords] tiles, staged in place
    static constexpr uint32_t kCnt = kIn + 2u * kInWords;           // [kSeg * kThreads] counters
    static constexpr uint32_t kPieces = kCnt + kSeg * kThreads;     // [kMaxPieces] slot - stage position
    static constexpr uint32_t kBm = kPieces + kMaxPieces;           // [kBmWords] stage positions where pieces start
    // phase 1 and plan: [64] each; in phase 2 the four arrays hold the per-port chunk cache
    static constexpr uint32_t kBase = kBm + kBmWords;               // [64] this CTA's first port position
    static constexpr uint32_t kTotal = kBase + kBM;                 // [64] batch totals
    static constexpr uint32_t kOwn = kTotal + kBM;                  // [64] this CTA's totals
    static constexpr uint32_t kAcc = kOwn + kBM;                    // [64] phase-1 flushed counts
    static constexpr uint32_t kChunkCache = kBase;                  // [64] x uint4 {k, id of chunk k, id of k + 1, -}
    static constexpr uint32_t kBinBase = kAcc + kBM;                // [64] dense plan
    static constexpr uint32_t kScan = kBinBase + kBM;               // [kWarps]
    static constexpr uint32_t kTiles = kScan + 4u;                  // [4][4] tile descriptors (phase 1, phase 2)
    static constexpr uint32_t kMisc = kTiles + 16u;                 // [8]
    static constexpr uint32_t kMbar = kMisc + 8u;                   // [2] x u64
    static constexpr uint32_t kWords = kMbar + 4u;
    static constexpr size_t kSmemBytes = sizeof(uint32_t) * kWords;
    static_assert(kCnt % 4u == 0u && kChunkCache % 4u == 0u && kMbar % 2u == 0u, "alignment");
    static_assert(kWarps == 4 && kMaxCount == (uint32_t)kWarps * 1024u, "write-out: one 1024-position quarter per warp");
};

// Grid-wide barrier of a cooperative launch on a counter reset before the launch. Bounded: a wait
// that gives up sets GF_ERR_TIMEOUT and returns.
GF_D void coop_grid_barrier(unsigned long long* counter, uint32_t* status)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(counter, 1ull);
        uint32_t polls = 0;
        while (ld_acquire_u64(counter) < gridDim.x) {
            if (++polls >= g_spin_limit) {
                set_status(status, GF_ERR_TIMEOUT);
                break;
            }
            __nanosleep(polls < 64u ? 32u : 128u);
        }
        __threadfence();
    }
    __syncthreads();
}

// Thread 0: fetch `tile` into the shared buffer at word offset `dst` (bulk copy completing on
// `bar`, or a plain arrival when the tile cannot be bulk copied) and describe it in d[0..3]:
// chunk, offset, count (0 for an invalid tile), flags (1 = valid, 2 = in shared memory). The
// caller loads the tile's descriptor ahead of time, so its global-memory latency overlaps work.
GF_D void coop_fetch(const gf_tile tile, const uint32_t* in, uint32_t capacity, uint64_t pool_slots,
                     uint32_t max_count, uint32_t* sm, uint32_t dst, uint64_t* bar, uint32_t* d, uint32_t* status)
{
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
__global__ void __launch_bounds__(S::kThreads, 4)
    fused_partition_coop_kernel(const uint32_t* __restrict__ in, uint32_t* out, Classify cls, uint32_t capacity,
                                FastDiv fdc, uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t B,
                                const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                                unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl, CoopHdr* hdr,
                                uint32_t* cta_tot, uint32_t* status, InlineFinish fin)
{
    constexpr int T = S::kThreads, IPT = S::kIpt, W = S::kWarps;
    constexpr uint32_t BM = S::kBM, L = S::kLanes, SEG = S::kSeg, MB = S::kMaxBins;
    constexpr bool kValid = always_valid<Classify>();
    extern __shared__ __align__(128) uint32_t sm[];
    uint32_t* cnt = sm + S::kCnt;
    uint16_t* cnt16 = reinterpret_cast<uint16_t*>(cnt);
    uint32_t* pieces = sm + S::kPieces;
    uint32_t* bm = sm + S::kBm;
    uint32_t* cbase = sm + S::kBase;
    uint32_t* total = sm + S::kTotal;
    uint32_t* bin_base = sm + S::kBinBase;
    uint32_t* own = sm + S::kOwn;
    uint32_t* acc = sm + S::kAcc;
    uint4* ccache = reinterpret_cast<uint4*>(sm + S::kChunkCache);
    uint32_t* scan = sm + S::kScan;
    uint32_t* tdesc = sm + S::kTiles;
    uint32_t* misc = sm + S::kMisc;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + S::kMbar);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    auto buffer = [](uint32_t buf) { return S::kIn + buf * S::kInWords; };

    // this CTA's tiles: [t_lo, t_hi) of an even split
    const uint32_t t_lo = (uint32_t)((uint64_t)n_tiles * c / G);
    const uint32_t t_hi = (uint32_t)((uint64_t)n_tiles * (c + 1u) / G);
    const uint32_t n_mine = t_hi - t_lo;
    if (tid == 0) {
        misc[0] = next_epoch(ld_relaxed_u32(&ctl->epoch));
        mbar_init(&mbar[0], 1u);
        mbar_init(&mbar[1], 1u);
        mbar_init_fence();
    }
    for (uint32_t i = tid; i < SEG * T; i += T)
        cnt[i] = 0u;
    if (tid < BM)
        acc[tid] = 0u;
    __syncthreads();
    const uint32_t epoch = misc[0];

    // ---------------- phase 1: per-port counts of this CTA's tiles (forward, two buffers) ----------------
    if (tid == 0)
        for (uint32_t q = 0; q < 2u && q < n_mine; ++q)
            coop_fetch(tiles[t_lo + q], in, capacity, pool_slots, S::kMaxCount, sm, buffer(q), &mbar[q],
                       tdesc + 4u * q, status);
    bool bad = false;
    auto count_key = [&](uint32_t key) {
        const uint32_t b = cls(key);
        if (kValid || b < B) // own column: no contention; a reduction, so consecutive keys do not wait on each other
            atomicAdd(cnt + (b & (L - 1u)) * T + tid, 1u << ((b >> S::kLaneShift) << 4));
        else
            bad = true;
    };
    // adds the packed counters into acc[] and clears them (a thread counts at most 32 keys per tile,
    // so 1024 tiles between flushes keep every 16-bit counter at or below 2^15)
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
        const uint32_t buf = q & 1u;
        const uint32_t* d = tdesc + 4u * buf;
        gf_tile next{};
        if (tid == 0 && q + 2u < n_mine)
            next = tiles[t_lo + q + 2u]; // used after this tile's barrier
        mbar_wait(&mbar[buf], (q >> 1) & 1u, status);
        const uint32_t count = d[2], flags = d[3];
        if ((flags & 2u) && count == S::kMaxCount) { // a full tile: no per-key checks
            const uint4* v = reinterpret_cast<const uint4*>(sm + buffer(buf));
#pragma unroll
            for (uint32_t j = 0; j < S::kMaxCount / 4u / (uint32_t)T; ++j) {
                const uint4 x = v[tid + j * (uint32_t)T];
                count_key(x.x);
                count_key(x.y);
                count_key(x.z);
                count_key(x.w);
            }
        } else if (flags & 2u) {
            const uint4* v = reinterpret_cast<const uint4*>(sm + buffer(buf));
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
        if (tid == 0 && q + 2u < n_mine)
            coop_fetch(next, in, capacity, pool_slots, S::kMaxCount, sm, buffer(buf), &mbar[buf],
                       tdesc + 4u * buf, status);
        if ((q & 1023u) == 1023u)
            flush();
    }
    if (bad)
        set_status(status, GF_INVALID);
    flush();
    if (tid < BM) {
        const uint32_t v = tid < B ? acc[tid] : 0u;
        own[tid] = v;
        if (tid < MB) {
            cta_tot[(size_t)c * MB + tid] = v << 2; // see CoopHdr: v < 2^30 (checked by the launcher)
            if (v != 0u)
                atomicAdd(&hdr->total[tid], (unsigned long long)v);
        }
    }
    // phase 2 walks the tiles last to first through the same two buffers; its first two tiles are
    // fetched across the barrier. Uses of each buffer so far set the mbarrier parities.
    const uint32_t use0 = (n_mine + 1u) / 2u, use1 = n_mine / 2u;
    if (tid == 0)
        for (uint32_t k = 0; k < 2u && k < n_mine; ++k)
            coop_fetch(tiles[t_hi - 1u - k], in, capacity, pool_slots, S::kMaxCount, sm, buffer(k), &mbar[k],
                       tdesc + 8u + 4u * k, status);

    coop_grid_barrier(&hdr->done, status);

    // ---------------- plan ----------------
    {
        // this CTA's per-port base from the fewer of the rows before it and the rows after it:
        // thread tid sums ports [4 qd, 4 qd + 4) of rows g, g + NG, ... with 128-bit loads
        constexpr uint32_t QUADS = MB / 4u, NG = (uint32_t)T / QUADS;
        const uint32_t qd = tid % QUADS, g = tid / QUADS;
        const bool before = c <= G - 1u - c;
        const uint32_t r_lo = before ? 0u : c + 1u, r_hi = before ? c : G;
        uint4 s = make_uint4(0u, 0u, 0u, 0u);
        for (uint32_t r0 = r_lo + g; r0 < r_hi; r0 += NG * 8u) {
            uint4 v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const uint32_t rr = r0 + (uint32_t)u * NG;
                v[u] = rr < r_hi ? __ldcg(reinterpret_cast<const uint4*>(cta_tot + (size_t)rr * MB) + qd)
                                 : make_uint4(0u, 0u, 0u, 0u);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                s.x += v[u].x >> 2;
                s.y += v[u].y >> 2;
                s.z += v[u].z >> 2;
                s.w += v[u].w >> 2;
            }
        }
        uint4* red = reinterpret_cast<uint4*>(cnt); // the counters are zero now and are zeroed again below
        red[tid] = s;
        __syncthreads();
        if (tid < BM) {
            uint32_t part = 0;
            if (tid < MB) {
                const uint32_t q = tid >> 2, e = tid & 3u;
                for (uint32_t g2 = 0; g2 < NG; ++g2) {
                    const uint4 x = red[g2 * QUADS + q];
                    part += e == 0u ? x.x : e == 1u ? x.y : e == 2u ? x.z : x.w;
                }
            }
            const uint32_t tot = tid < B ? (uint32_t)ld_relaxed_u64(&hdr->total[tid]) : 0u;
            total[tid] = tot;
            cbase[tid] = tid < B ? (before ? part : tot - own[tid] - part) : 0u;
        }
        __syncthreads();
        red[tid] = make_uint4(0u, 0u, 0u, 0u);
        if (w == 0) {
            // binBase = exclusive scan of ceil(total / C) (two ports per lane)
            const uint32_t b0 = 2u * lane, b1 = b0 + 1u;
            uint32_t n0 = 0, n1 = 0;
            if (b0 < B)
                n0 = fdc.div(total[b0]) + (fdc.mod(total[b0]) != 0u ? 1u : 0u);
            if (b1 < B)
                n1 = fdc.div(total[b1]) + (fdc.mod(total[b1]) != 0u ? 1u : 0u);
            uint32_t incl = n0 + n1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                if ((int)lane >= o)
                    incl += y;
            }
            const uint32_t ex = incl - n0 - n1;
            bin_base[b0] = ex;
            bin_base[b1] = ex + n0;
            if (lane == 31) {
                misc[1] = incl; // R = chunks of the plan
                if (incl > n_reserved)
                    set_status(status, GF_OVERFLOW);
            }
        }
        __syncthreads();
        const uint32_t R = misc[1];
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
        if (fin.table != nullptr) {
            // the finish, spread over the grid: output chunk r of the plan is reserved[r]; its port is
            // the last one whose chunks start at or before r (table = [binBase, chunkIndex],
            // DenseBinTable.hpp:80-91; descriptors in bin order with fills, Execution.hpp:2558-2581)
            for (uint32_t r = c * (uint32_t)T + tid; r < R; r += G * (uint32_t)T) {
                if (r >= fin.desc_cap) {
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
                const uint32_t chunk = r < n_reserved ? __ldg(reserved + r) : kNoChunk;
                fin.table[B + r] = chunk;
                fin.descs[r].chunk_index = chunk;
                fin.descs[r].fill = min(capacity, total[lo] - k * capacity);
                fin.descs[r].bin = lo;
            }
            if (c == 0) {
                for (uint32_t b2 = tid; b2 < B; b2 += T)
                    fin.table[b2] = bin_base[b2];
                if (tid == 0)
                    *fin.num_out = R;
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
    if (misc[2] != 0u) {
        // a failed batch writes nothing: wait for this CTA's two phase-2 copies, then leave
        if (tid == 0)
            for (uint32_t k = 0; k < 2u && k < n_mine; ++k)
                mbar_wait(&mbar[k], (k == 0u ? use0 : use1) & 1u, status);
        return;
    }
    const uint32_t R = misc[1];

    // chunk id of port b's k-th output chunk
    auto chunk_of = [&](uint32_t b, uint32_t k) -> uint32_t {
        const uint32_t f = bin_base[b] + k;
        return f < R && f < n_reserved ? __ldg(reserved + f) : kNoChunk;
    };
    // a chunk id outside the pool writes nothing and fails the batch
    const uint32_t pool_chunks = (uint32_t)(pool_slots / capacity); // < 2^20: pool_slots < 2^32, C >= 4096
    auto in_pool = [&](uint32_t ch) {
        const bool okc = ch < pool_chunks; // kNoChunk is never below it
        if (!okc)
            set_status(status, GF_OVERFLOW);
        return okc;
    };

    // warp 0 keeps the running port positions (two ports per lane): the end of this CTA's range,
    // since its tiles are walked last to first
    uint32_t off0 = 0, off1 = 0;
    if (w == 0) {
        off0 = cbase[2u * lane] + own[2u * lane];
        off1 = cbase[2u * lane + 1u] + own[2u * lane + 1u];
    }
    __syncthreads(); // the plan's per-port arrays are read; their words become the chunk cache
    // per port: the two chunks its last run touched (walking backwards, the next run touches the
    // same pair or the pair below), so a tile's pieces rarely reach for the reservation itself
    if (tid < BM)
        ccache[tid] = make_uint4(0xFFFFFFFFu, kNoChunk, kNoChunk, 0u);

    // ---------------- phase 2: rank, stage, write (tiles last to first) ----------------
    for (uint32_t k = 0; k < n_mine; ++k) {
        const uint32_t buf = k & 1u;
        const uint32_t* d = tdesc + 8u + 4u * buf;
        uint32_t* tin = sm + buffer(buf);
        gf_tile next{};
        if (tid == 0 && k >= 1u && k + 1u < n_mine)
            next = tiles[t_hi - 2u - k]; // used after this tile's first barrier
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
        // count: a key's local rank is its 16-bit counter before the increment (the atomics of one
        // thread are independent instructions, so they issue back to back); a slot past the tile's
        // count adds 0 (its key is never staged)
        // pk: byte offset of the key's 16-bit counter (low half) and its local rank (high half)
        uint32_t pk[IPT];
        // every slot of every thread of this warp holds a key (uniform per warp: a warp with a few
        // short threads takes the checked path once instead of both paths)
        const bool full = __all_sync(0xFFFFFFFFu, tid * IPT + IPT <= count);
        auto count_keys = [&](auto all) {
#pragma unroll
            for (int i = 0; i < IPT; ++i) {
                const uint32_t valid = decltype(all)::value || tid * IPT + (uint32_t)i < count ? 1u : 0u;
                uint32_t b = cls(key[i]);
                if constexpr (!kValid)
                    b = b < B ? b : 0u;
                const uint32_t wi = (b & (L - 1u)) * T + tid;
                const uint32_t half = b >> S::kLaneShift;
                const uint32_t old = atomicAdd(cnt + wi, valid << (half << 4));
                pk[i] = __byte_perm((wi << 2) | (half << 1), old, half != 0u ? 0x7610u : 0x5410u);
            }
        };
        if (full)
            count_keys(std::true_type{});
        else
            count_keys(std::false_type{});
        __syncthreads();
        // the other buffer's last reader (the previous tile's write-out) is done: fetch the next tile
        if (tid == 0 && k >= 1u && k + 1u < n_mine)
            coop_fetch(next, in, capacity, pool_slots, S::kMaxCount, sm, buffer(buf ^ 1u),
                       &mbar[buf ^ 1u], tdesc + 8u + 4u * (buf ^ 1u), status);

        // raking scan over the (row, thread) counters: segments of SEG words, 128-bit accesses
        uint4* seg = reinterpret_cast<uint4*>(cnt + tid * SEG);
        uint32_t sum = 0;
#pragma unroll
        for (uint32_t j = 0; j < SEG / 4u; ++j) {
            const uint4 x = seg[j];
            sum += x.x + x.y + x.z + x.w;
        }
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
        // words past the L counter rows stay zero (the per-column reset below clears only L rows)
#pragma unroll
        for (uint32_t j = 0; j < SEG / 4u; ++j) {
            const uint4 x = seg[j];
            uint4 y;
            y.x = run;
            y.y = y.x + x.x;
            y.z = y.y + x.y;
            y.w = y.z + x.z;
            run = y.w + x.w;
            if (tid * SEG + 4u * j < L * (uint32_t)T)
                seg[j] = y;
        }
        __syncthreads();

        // warp 0: each port's run [s, s + len) in the stage is cut at its output-chunk boundary into
        // at most two pieces; piece i (in stage order) gets {slot - stage position, ok} and a bit at
        // its first stage position
        if (w == 0) {
#pragma unroll
            for (uint32_t i = lane; i < S::kBmWords; i += 32u)
                bm[i] = 0u;
            const uint32_t b0 = 2u * lane, b1 = b0 + 1u;
            auto start_of = [&](uint32_t b) -> uint32_t {
                return b < MB ? (uint32_t)cnt16[(((b & (L - 1u)) * T) << 1) | (b >> S::kLaneShift)] : count;
            };
            const uint32_t s0 = start_of(b0), s1 = start_of(b1), s2 = start_of(b1 + 1u);
            uint32_t ps[4], pl[4], pb[4], pv[4];
            auto cut = [&](uint32_t b, uint32_t s, uint32_t len, uint32_t& off, int p) {
                pl[p] = pl[p + 1] = 0u;
                ps[p] = ps[p + 1] = pb[p] = pb[p + 1] = pv[p] = pv[p + 1] = 0u;
                if (b >= B || len == 0u)
                    return;
                const uint32_t j0 = off - len;
                off = j0;
                const uint32_t k0 = fdc.div(j0);
                const uint32_t room = (k0 + 1u) * capacity - j0; // slots left in the first chunk
                const uint32_t n1 = len < room ? len : room;
                uint4 cc = ccache[b];
                if (cc.x != k0) {
                    cc = make_uint4(k0, chunk_of(b, k0), chunk_of(b, k0 + 1u), 0u);
                    ccache[b] = cc;
                }
                const uint32_t ca = cc.y;
                ps[p] = s;
                pl[p] = n1;
                pv[p] = in_pool(ca) ? 1u : 0u;
                pb[p] = ca * capacity + (j0 - k0 * capacity) - s;
                if (len > room) {
                    const uint32_t cb = cc.z;
                    ps[p + 1] = s + n1;
                    pl[p + 1] = len - n1;
                    pv[p + 1] = in_pool(cb) ? 1u : 0u;
                    pb[p + 1] = cb * capacity - (s + n1);
                }
            };
            cut(b0, s0, s1 - s0, off0, 0);
            cut(b1, s1, s2 - s1, off1, 2);
            const uint32_t n_p = (pl[0] != 0u) + (pl[1] != 0u) + (pl[2] != 0u) + (pl[3] != 0u);
            // exclusive prefix of the lanes' piece counts (0..4): one ballot per bit
            const uint32_t below = lanemask_lt();
            uint32_t at = 0;
#pragma unroll
            for (int bit = 0; bit < 3; ++bit)
                at += (uint32_t)__popc(__ballot_sync(0xFFFFFFFFu, (n_p >> bit) & 1u) & below) << bit;
            bool ok = true;
#pragma unroll
            for (int p = 0; p < 4; ++p)
                ok = ok && (pl[p] == 0u || pv[p] != 0u);
            ok = __all_sync(0xFFFFFFFFu, ok);
            __syncwarp();
#pragma unroll
            for (int p = 0; p < 4; ++p)
                if (pl[p] != 0u && at < S::kMaxPieces) {
                    pieces[at++] = pb[p];
                    atomicOr(&bm[ps[p] >> 5], 1u << (ps[p] & 31u));
                }
            if (lane == 0u)
                misc[4] = ok ? 1u : 0u; // a piece outside the pool has failed the batch: the tile writes nothing
            __syncwarp();
        }

        // stage in port order (the stage position is the rank) in this tile's own buffer: its keys
        // are in registers. All positions are read before any key is stored.
        const char* cbytes = reinterpret_cast<const char*>(cnt);
#pragma unroll
        for (int i = 0; i < IPT; ++i)
            pk[i] = *reinterpret_cast<const uint16_t*>(cbytes + (pk[i] & 0xFFFFu)) + (pk[i] >> 16);
        if (full) {
#pragma unroll
            for (int i = 0; i < IPT; ++i)
                tin[pk[i]] = key[i];
        } else {
#pragma unroll
            for (int i = 0; i < IPT; ++i)
                if (tid * IPT + (uint32_t)i < count)
                    tin[pk[i]] = key[i];
        }
        // this thread's counter column is reset for the next tile (no other thread reads it now)
#pragma unroll
        for (uint32_t r = 0; r < L; ++r)
            cnt[r * T + tid] = 0u;
        __syncthreads();

        // write-out: warp w covers stage positions [1024 w, 1024 w + 1024) in windows of 32, lane =
        // position within the window; a position's piece is the last piece starting at or before it
        if (misc[4] != 0u) {
            uint32_t kb = 0; // pieces starting before this warp's first window
            for (uint32_t i = lane; i < w * 32u; i += 32u)
                kb += __popc(bm[i]);
            kb = __reduce_add_sync(0xFFFFFFFFu, kb);
            const uint32_t upto = 0xFFFFFFFFu >> (31u - lane);
            const uint32_t* pcs = pieces - 1; // indexed by the number of piece starts at or before q
            auto write_out = [&](auto all) {
#pragma unroll
                for (uint32_t i0 = 0; i0 < 32u; i0 += 8u) {
                    uint32_t wd[8], v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const uint32_t win = w * 32u + i0 + (uint32_t)u;
                        wd[u] = bm[win];
                        v[u] = tin[win * 32u + lane];
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const uint32_t q = (w * 32u + i0 + (uint32_t)u) * 32u + lane;
                        const uint32_t kk = kb + __popc(wd[u] & upto);
                        kb += __popc(wd[u]);
                        if (decltype(all)::value || q < count)
                            out[q + pcs[kk]] = v[u]; // 32-bit slot arithmetic: the base wraps, the slot does not
                    }
                }
            };
            if (count == S::kMaxCount)
                write_out(std::true_type{});
            else
                write_out(std::false_type{});
        }
        fence_proxy_async_smem(); // this buffer's reads come before the next bulk copy into it
    }
}

// Host side: one cooperative launch of the kernel with classifier `cls`; the grid is as many CTAs
// as fit on the device at once, capped by the tiles and by the scratch (the control block, then
// 4 * 2 * LANES bytes per CTA); a batch whose CTAs would own 2^30 keys or more is refused. The
// control block is zeroed here, on the stream.
// With `fin` set, the launch also writes the chunk table, descriptors and output count.
template <typename S, typename Cls>
cudaError_t launch_fused_coop(cudaStream_t stream, Cls cls, const uint32_t* in, uint32_t* out, uint32_t capacity,
                              uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t bins,
                              const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                              unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl, uint64_t scratch_bytes,
                              uint32_t* status, int sms, InlineFinish fin = {})
{
    auto kernel = fused_partition_coop_kernel<S, Cls>;
    constexpr uint64_t kHead = sizeof(FusedCtl) + sizeof(CoopHdr);
    constexpr uint64_t kRow = sizeof(uint32_t) * S::kMaxBins;
    if (scratch_bytes < kHead + kRow)
        return cudaErrorInvalidValue;
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
    const uint64_t cap_ctas = (scratch_bytes - kHead) / kRow;
    g = g < cap_ctas ? g : cap_ctas;
    if (g == 0u)
        return cudaErrorInvalidConfiguration;
    // every CTA owns at most ceil(n_tiles / g) tiles of at most kMaxCount keys: below 2^30 (CoopHdr)
    if (((uint64_t)n_tiles + g - 1u) / g * S::kMaxCount >= (1ull << 30))
        return cudaErrorInvalidConfiguration;
    CoopHdr* hdr = reinterpret_cast<CoopHdr*>(ctl + 1);
    uint32_t* cta_tot = reinterpret_cast<uint32_t*>(hdr + 1);
    err = cudaMemsetAsync(hdr, 0, kCoopHdrResetBytes, stream);
    if (err != cudaSuccess)
        return err;
    FastDiv fd(capacity);
    void* args[] = {&in,       &out,      &cls,    &capacity,    &fd,    &pool_slots, &tiles,
                    &n_tiles,  &bins,     &reserved, &n_reserved, &totals, &port_chunks, &max_k,
                    &ctl,      &hdr,      &cta_tot, &status, &fin};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3((uint32_t)g), dim3(S::kThreads),
                                       args, S::kSmemBytes, stream);
}

} // namespace
} // namespace gf
