// Cooperative dense partition with a bulk-copy write-out, for u32 keys and up to 16 ports.
//
// Same contract and results as fused_partition_coop_kernel (gf_fused_coop.cuh): per-port totals,
// the exact plan and every port's keys in input order. What differs is how a tile reaches memory.
// With few ports a tile's keys form a few long runs, and each run is written by the bulk-copy
// (TMA) engine instead of warp stores:
//   phase 1  as the other kernel, plus each tile's per-port histogram (8-bit counters, four ports
//            per word, in two alternating matrices so the flush of one tile overlaps the count of
//            the next) written to the scratch (16-bit counts times four, 4 x LANES bytes per tile);
//   plan     as the other kernel;
//   phase 2  tiles last to first: the tile arrives with its histogram (bulk copies); warp 0 turns
//            the histogram into port runs, each run's output slot and its cut at the output-chunk
//            boundary (at most two pieces), and a stage layout padded so that every piece starts
//            at the same address modulo 16 bytes as its output slots; the pads enter the raking
//            scan as counts of the last thread column; keys are ranked and staged as in the other
//            kernel; one thread per piece then copies its 16-byte aligned body with
//            cp.async.bulk (global <- shared) and up to three slots either side with plain stores.
// Requirements (checked by the dispatcher): B <= 16, tiles of at most 4096 keys, capacity % 4 == 0
// and >= 4096, fewer than 2^32 pool slots, key columns 16-byte aligned, scratch for the control
// block, 4 * B_max bytes per CTA and the per-tile histograms.
#pragma once

#include "gf_fused_coop.cuh"

namespace gf {
namespace {

// 1-D bulk copy shared -> global of `bytes` (multiple of 16, both addresses 16-byte aligned) into
// this thread's current bulk group.
GF_D void bulk_store(void* gdst, const void* ssrc, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(ssrc)),
                 "r"(bytes)
                 : "memory");
}
// Bulk groups of this thread: close the open one; wait until all have read their shared-memory
// source (.read) or have completed.
GF_D void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
GF_D void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
GF_D void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's generic-proxy memory accesses before later async-proxy (bulk copy) ones.
GF_D void fence_proxy_async_all() { asm volatile("fence.proxy.async;" ::: "memory"); }

// 128 threads, 33 keys each; LANES counter rows with two 16-bit port counters per word (up to
// 2 * LANES ports, LANES = 2 or 8).
template <int LANES>
struct CoopBulkShape {
    static_assert(LANES == 2 || LANES == 8, "2 or 8 counter rows");
    static constexpr int kThreads = 128;
    static constexpr int kWarps = 4;
    static constexpr int kIpt = 33;
    static constexpr uint32_t kMaxCount = 4096u;
    static constexpr uint32_t kInWords = (uint32_t)kThreads * kIpt; // 4224
    static constexpr uint32_t kLanes = LANES;
    static constexpr uint32_t kLaneShift = LANES == 2 ? 1u : (LANES == 8 ? 3u : 5u);
    static constexpr uint32_t kMaxBins = 2u * LANES;
    static constexpr uint32_t kBM = 64u;
    static constexpr uint32_t kSeg = LANES == 2 ? 4u : LANES + 4u;
    static constexpr uint32_t kHistWords = LANES < 4 ? 4u : LANES; // one tile's histogram (16-byte multiple)
    static constexpr uint32_t kStageWords = (kMaxCount + 3u * kMaxBins + 31u) & ~31u;
    // shared memory (32-bit words)
    static constexpr uint32_t kIn = 0;                             // phase 1 buffer 0, phase 2 input
    static constexpr uint32_t kHist = kIn + kInWords;              // phase 2: this tile's histogram
    static constexpr uint32_t kStage = kHist + kHistWords;         // phase 1 buffer 1, phase 2 stage
    static constexpr uint32_t kCnt = kStage + kStageWords;         // [kSeg * kThreads] counters
    static constexpr uint32_t kInj = kCnt + kSeg * kThreads;       // [LANES] scan injections
    static constexpr uint32_t kBase = kInj + (LANES < 4 ? 4u : LANES);
    static constexpr uint32_t kTotal = kBase + kBM;
    static constexpr uint32_t kOwn = kTotal + kBM;
    static constexpr uint32_t kAcc = kOwn + kBM;
    static constexpr uint32_t kBinBase = kAcc + kBM;
    static constexpr uint32_t kScan = kBinBase + kBM;
    static constexpr uint32_t kTiles = kScan + 4u; // [3][4]
    static constexpr uint32_t kMisc = kTiles + 12u;
    static constexpr uint32_t kMbar = kMisc + 8u; // [3] x u64
    static constexpr uint32_t kPc = kMbar + 8u;    // [2 * kMaxBins] x uint4 pieces {slot, stage pos, n, -}
    static constexpr uint32_t kWords = kPc + 8u * kMaxBins;
    static constexpr size_t kSmemBytes = sizeof(uint32_t) * kWords;
    static_assert(kPc % 4u == 0u && kHist % 4u == 0u && kStage % 4u == 0u && kCnt % 4u == 0u && kMbar % 2u == 0u,
                  "alignment");
    static_assert(kStageWords >= kMaxCount, "stage doubles as a phase-1 buffer");
};

// Thread 0: fetch `tile` (and, with `hist`, its histogram) into shared memory, completing on `bar`.
GF_D void coop_bulk_fetch(const gf_tile tile, const uint32_t* in, uint32_t capacity, uint64_t pool_slots,
                          uint32_t max_count, uint32_t* sm, uint32_t dst, const uint32_t* hist, uint32_t hist_dst,
                          uint32_t hist_words, uint64_t* bar, uint32_t* d, uint32_t* status)
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
    const uint32_t hb = hist != nullptr ? hist_words * 4u : 0u;
    const uint32_t tb = bulk ? words * 4u : 0u;
    if (hb + tb != 0u) {
        mbar_expect_tx(bar, hb + tb);
        if (tb)
            bulk_load(sm + dst, in + base, tb, bar);
        if (hb)
            bulk_load(sm + hist_dst, hist, hb, bar);
    } else {
        mbar_arrive(bar);
    }
}

// The kernel: one cooperative launch over all tiles of the batch (layout of the scratch at
// launch_fused_coop_bulk).
template <typename S, typename Classify>
__global__ void __launch_bounds__(S::kThreads, 4)
    fused_partition_coop_bulk_kernel(const uint32_t* __restrict__ in, uint32_t* out, Classify cls, uint32_t capacity,
                                     FastDiv fdc, uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles,
                                     uint32_t B, const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                                     unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl, CoopHdr* hdr,
                                     uint32_t* cta_tot, uint32_t* tile_hist, uint32_t* status, InlineFinish fin)
{
    constexpr int T = S::kThreads, IPT = S::kIpt, W = S::kWarps;
    constexpr uint32_t BM = S::kBM, L = S::kLanes, SEG = S::kSeg, MB = S::kMaxBins, HW = S::kHistWords;
    constexpr bool kValid = always_valid<Classify>();
    extern __shared__ __align__(128) uint32_t sm[];
    uint32_t* cnt = sm + S::kCnt;
    uint32_t* stage = sm + S::kStage;
    uint32_t* hist = sm + S::kHist;
    uint32_t* inj = sm + S::kInj;
    uint32_t* cbase = sm + S::kBase;
    uint32_t* total = sm + S::kTotal;
    uint32_t* bin_base = sm + S::kBinBase;
    uint32_t* own = sm + S::kOwn;
    uint32_t* acc = sm + S::kAcc;
    uint32_t* scan = sm + S::kScan;
    uint32_t* tdesc = sm + S::kTiles;
    uint32_t* misc = sm + S::kMisc;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + S::kMbar);
    uint4* pcs = reinterpret_cast<uint4*>(sm + S::kPc);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    auto buffer1 = [](uint32_t buf) { return buf == 0u ? S::kIn : S::kStage; };

    const uint32_t t_lo = (uint32_t)((uint64_t)n_tiles * c / G);
    const uint32_t t_hi = (uint32_t)((uint64_t)n_tiles * (c + 1u) / G);
    const uint32_t n_mine = t_hi - t_lo;
    if (tid == 0) {
        misc[0] = next_epoch(ld_relaxed_u32(&ctl->epoch));
        mbar_init(&mbar[0], 1u);
        mbar_init(&mbar[1], 1u);
        mbar_init(&mbar[2], 1u);
        mbar_init_fence();
    }
    for (uint32_t i = tid; i < SEG * T; i += T)
        cnt[i] = 0u;
    if (tid < BM)
        acc[tid] = 0u;
    __syncthreads();
    const uint32_t epoch = misc[0];

    // ---------------- phase 1: per-tile histograms and this CTA's per-port counts ----------------
    // 8-bit counters, four ports per word (row b % R1, byte b / R1; a thread counts at most 32 keys
    // of a tile) in two matrices: tile q counts into matrix q % 2, so the flush of a tile's matrix
    // overlaps the count of the next tile without a second barrier.
    constexpr uint32_t R1 = MB / 4u;                 // rows: 16, 4, 1
    constexpr uint32_t R1S = R1 == 16u ? 4u : (R1 == 4u ? 2u : 0u);
    constexpr uint32_t G1 = R1 >= 4u ? (uint32_t)T / R1 : 32u; // flushing threads per row: 8, 32, 32
    constexpr uint32_t WPT = (uint32_t)T / G1;                  // words per flushing thread: 16, 4, 4
    if (tid == 0)
        for (uint32_t q = 0; q < 2u && q < n_mine; ++q)
            coop_bulk_fetch(tiles[t_lo + q], in, capacity, pool_slots, S::kMaxCount, sm, buffer1(q), nullptr, 0u,
                            0u, &mbar[q], tdesc + 4u * q, status);
    bool bad = false;
    const uint32_t frow = tid / G1, fpart = tid % G1;
    uint32_t tel = 0, teh = 0, tol = 0, toh = 0; // flush leaders: running per-port totals of this CTA
    for (uint32_t q = 0; q < n_mine; ++q) {
        const uint32_t buf = q & 1u;
        uint32_t* mat = cnt + buf * R1 * (uint32_t)T;
        auto count_key = [&](uint32_t key) {
            const uint32_t b = cls(key);
            if (kValid || b < B)
                atomicAdd(mat + (b & (R1 - 1u)) * T + tid, 1u << ((b >> R1S) << 3));
            else
                bad = true;
        };
        const uint32_t* d = tdesc + 4u * buf;
        gf_tile next{};
        if (tid == 0 && q + 2u < n_mine)
            next = tiles[t_lo + q + 2u];
        mbar_wait(&mbar[buf], (q >> 1) & 1u, status);
        const uint32_t count = d[2], flags = d[3];
        const uint4* v = reinterpret_cast<const uint4*>(sm + buffer1(buf));
        if ((flags & 2u) && count == S::kMaxCount) {
#pragma unroll
            for (uint32_t j = 0; j < S::kMaxCount / 4u / (uint32_t)T; ++j) {
                const uint4 x = v[tid + j * (uint32_t)T];
                count_key(x.x);
                count_key(x.y);
                count_key(x.z);
                count_key(x.w);
            }
        } else if (flags & 2u) {
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
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0 && q + 2u < n_mine)
            coop_bulk_fetch(next, in, capacity, pool_slots, S::kMaxCount, sm, buffer1(buf), nullptr, 0u, 0u,
                            &mbar[buf], tdesc + 4u * buf, status);
        // flush: row r's even bytes are ports r and r + L, its odd bytes ports r + R1 and r + R1 + L,
        // i.e. histogram words r and r + R1 (16-bit halves; a row sums to at most 4096 per port).
        // Stored times four (see CoopHdr: the words read as unpublished look-back descriptors).
        if (frow < R1) {
            uint32_t ev = 0, od = 0;
            uint4* row = reinterpret_cast<uint4*>(mat + frow * T + fpart * WPT);
#pragma unroll
            for (uint32_t j = 0; j < WPT / 4u; ++j) {
                const uint32_t jj = WPT == 16u ? ((j + (fpart >> 1)) & 3u) : j; // distinct bank groups
                const uint4 x = row[jj];
                row[jj] = make_uint4(0u, 0u, 0u, 0u);
                ev += (x.x & 0x00FF00FFu) + (x.y & 0x00FF00FFu) + (x.z & 0x00FF00FFu) + (x.w & 0x00FF00FFu);
                od += ((x.x >> 8) & 0x00FF00FFu) + ((x.y >> 8) & 0x00FF00FFu) + ((x.z >> 8) & 0x00FF00FFu) +
                      ((x.w >> 8) & 0x00FF00FFu);
            }
#pragma unroll
            for (uint32_t o = 1; o < G1; o <<= 1) {
                ev += __shfl_xor_sync(0xFFFFFFFFu, ev, o);
                od += __shfl_xor_sync(0xFFFFFFFFu, od, o);
            }
            if (fpart == 0u) {
                uint32_t* th = tile_hist + (size_t)(t_lo + q) * HW;
                th[frow] = ev << 2;
                th[frow + R1] = od << 2;
                fence_proxy_async_all(); // the histogram stores come before this CTA's bulk reads of them
                tel += ev & 0xFFFFu;
                teh += ev >> 16;
                tol += od & 0xFFFFu;
                toh += od >> 16;
            }
        }
    }
    if (frow < R1 && fpart == 0u) {
        acc[frow] = tel;
        acc[frow + L] = teh;
        acc[frow + R1] = tol;
        acc[frow + R1 + L] = toh;
    }
    __syncthreads();
    if (bad)
        set_status(status, GF_INVALID);
    if (tid < BM) {
        const uint32_t v = tid < B ? acc[tid] : 0u;
        own[tid] = v;
        if (tid < MB) {
            cta_tot[(size_t)c * MB + tid] = v << 2;
            if (v != 0u)
                atomicAdd(&hdr->total[tid], (unsigned long long)v);
        }
    }
    // phase 2's first tile (the last one) is fetched across the barrier
    if (tid == 0 && n_mine != 0u)
        coop_bulk_fetch(tiles[t_hi - 1u], in, capacity, pool_slots, S::kMaxCount, sm, S::kIn,
                        tile_hist + (size_t)(t_hi - 1u) * HW, S::kHist, HW, &mbar[2], tdesc + 8u, status);

    coop_grid_barrier(&hdr->done, status);

    // ---------------- plan (as fused_partition_coop_kernel) ----------------
    {
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
        uint4* red = reinterpret_cast<uint4*>(cnt);
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
                misc[1] = incl;
                if (incl > n_reserved)
                    set_status(status, GF_OVERFLOW);
            }
        }
        __syncthreads();
        const uint32_t R = misc[1];
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
                atomicExch(&ctl->epoch, epoch);
        }
        if (tid == 0)
            misc[2] = ld_relaxed_u32(status);
        __syncthreads();
    }
    if (misc[2] != 0u) {
        if (tid == 0 && n_mine != 0u)
            mbar_wait(&mbar[2], 0u, status);
        return;
    }
    const uint32_t R = misc[1];
    auto chunk_of = [&](uint32_t b, uint32_t k) -> uint32_t {
        const uint32_t f = bin_base[b] + k;
        return f < R && f < n_reserved ? __ldg(reserved + f) : kNoChunk;
    };
    const uint32_t pool_chunks = (uint32_t)(pool_slots / capacity);

    // warp 0, lane r: ports r (A) and r + L (B) while r < L: running end positions (tiles are walked
    // last to first), the two chunks the last run touched, and this tile's pieces
    uint32_t offA = 0, offB = 0;
    uint32_t ckA = 0xFFFFFFFFu, c0A = kNoChunk, c1A = kNoChunk, ckB = 0xFFFFFFFFu, c0B = kNoChunk, c1B = kNoChunk;
    const uint32_t pA = lane, pB = lane + L;
    if (w == 0 && lane < L) {
        if (pA < B)
            offA = cbase[pA] + own[pA];
        if (pB < B)
            offB = cbase[pB] + own[pB];
    }
    // the scan injection word this thread's raking segment holds (row r's last column), if any
    int inj_row = -1;
    {
        const uint32_t s0 = tid * SEG, s1 = s0 + SEG; // [s0, s1)
        if (s1 >= (uint32_t)T) {
            const uint32_t r = (s1 - (uint32_t)T) / (uint32_t)T; // largest r with r*T + T-1 < s1
            if (r * T + T - 1u >= s0 && r < L)
                inj_row = (int)r;
        }
    }
    __syncthreads();

    // ---------------- phase 2 ----------------
    for (uint32_t k = 0; k < n_mine; ++k) {
        const uint32_t* d = tdesc + 8u;
        uint32_t* tin = sm + S::kIn;
        gf_tile next{};
        if (tid == 0 && k + 1u < n_mine)
            next = tiles[t_hi - 2u - k];
        mbar_wait(&mbar[2], k & 1u, status);
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
        uint32_t pk[IPT];
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

        // warp 0: this tile's port runs from its histogram, their padded stage starts, the scan
        // injections and the pieces (a port's run cut at its output-chunk boundary)
        uint32_t pg[4], ps[4], pn[4];
        if (w == 0) {
            const uint32_t hw = lane < L ? hist[lane] >> 2 : 0u;
            const uint32_t lenA = pA < B ? hw & 0xFFFFu : 0u, lenB = pB < B ? hw >> 16 : 0u;
            uint32_t ia = lenA, ib = lenB;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t ya = __shfl_up_sync(0xFFFFFFFFu, ia, o);
                const uint32_t yb = __shfl_up_sync(0xFFFFFFFFu, ib, o);
                if ((int)lane >= o) {
                    ia += ya;
                    ib += yb;
                }
            }
            const uint32_t totA = __shfl_sync(0xFFFFFFFFu, ia, 31);
            const uint32_t uA = ia - lenA, uB = totA + ib - lenB; // unpadded starts
            const uint32_t jA = offA - lenA, jB = offB - lenB;
            offA = jA;
            offB = jB;
            // up to three pad slots before every port: its stage start is congruent to its first slot mod 4
            const uint32_t qA = uA + 3u * pA, qB = uB + 3u * pB;
            const uint32_t sA = qA + ((jA - qA) & 3u), sB = qB + ((jB - qB) & 3u);
            const uint32_t dA = sA - uA, dB = sB - uB;
            const uint32_t dA1 = __shfl_down_sync(0xFFFFFFFFu, dA, 1), dB1 = __shfl_down_sync(0xFFFFFFFFu, dB, 1);
            const uint32_t dB0 = __shfl_sync(0xFFFFFFFFu, dB, 0);
            if (lane < L) {
                // word (r, T-1) precedes port r+1 (low) and port r+L+1 (high) in scan order; the last
                // low word precedes the first high port
                const uint32_t lo = lane + 1u < L ? dA1 - dA : dB0 - dA;
                const uint32_t hi = lane + 1u < L ? dB1 - dB : 0u;
                inj[lane] = lo | (hi << 16);
            }
            if (lane == 0)
                misc[3] = dA; // D_0: offset of the whole stage
            bool ok = true;
            auto cut = [&](uint32_t b, uint32_t len, uint32_t j0, uint32_t s, uint32_t& ck, uint32_t& c0,
                           uint32_t& c1, int p) {
                pn[p] = pn[p + 1] = 0u;
                pg[p] = pg[p + 1] = ps[p] = ps[p + 1] = 0u;
                if (len == 0u)
                    return;
                const uint32_t k0 = fdc.div(j0);
                const uint32_t room = (k0 + 1u) * capacity - j0;
                const uint32_t n1 = len < room ? len : room;
                if (ck != k0) {
                    ck = k0;
                    c0 = chunk_of(b, k0);
                    c1 = chunk_of(b, k0 + 1u);
                }
                const bool v0 = c0 < pool_chunks;
                pg[p] = c0 * capacity + (j0 - k0 * capacity);
                ps[p] = s;
                pn[p] = n1;
                if (len > room) {
                    const bool v1 = c1 < pool_chunks;
                    pg[p + 1] = c1 * capacity;
                    ps[p + 1] = s + n1;
                    pn[p + 1] = len - n1;
                    ok = ok && v1;
                }
                ok = ok && v0;
            };
            cut(pA, lenA, jA, sA, ckA, c0A, c1A, 0);
            cut(pB, lenB, jB, sB, ckB, c0B, c1B, 2);
            ok = __all_sync(0xFFFFFFFFu, ok);
            if (!ok && lane == 0)
                set_status(status, GF_OVERFLOW);
            if (lane == 0)
                misc[4] = ok ? 1u : 0u;
        }
        fence_proxy_async_smem(); // this tile's reads of the input buffer come before the next bulk copy
        __syncthreads();
        if (tid == 0 && k + 1u < n_mine)
            coop_bulk_fetch(next, in, capacity, pool_slots, S::kMaxCount, sm, S::kIn,
                            tile_hist + (size_t)(t_hi - 2u - k) * HW, S::kHist, HW, &mbar[2], tdesc + 8u, status);
        // warp 0 lists this tile's pieces; the previous tile's write-out, their last reader, is done
        if (w == 0) {
            const uint32_t np = (pn[0] != 0u) + (pn[1] != 0u) + (pn[2] != 0u) + (pn[3] != 0u);
            uint32_t at = np;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, at, o);
                if ((int)lane >= o)
                    at += y;
            }
            if (lane == 31)
                misc[5] = at;
            at -= np;
#pragma unroll
            for (int p = 0; p < 4; ++p)
                if (pn[p] != 0u)
                    pcs[at++] = make_uint4(pg[p], ps[p], pn[p], 0u);
        }

        // raking scan over the (row, thread) counters with the injected padding
        if (inj_row >= 0)
            cnt[(uint32_t)inj_row * T + T - 1u] += inj[inj_row];
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
        uint32_t run = wpre + incl - sum + ((gtot & 0xFFFFu) << 16) + misc[3] * 0x10001u;
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
        bulk_wait_read0(); // the previous tile's stores have read the stage
        __syncthreads();
        // this tile's flag and piece count: warp 0 rewrites them for the next tile while the others
        // may still be writing this one out
        const uint32_t tile_ok = misc[4], n_pieces = misc[5];

        // stage in port order (padded layout)
        const char* cbytes = reinterpret_cast<const char*>(cnt);
#pragma unroll
        for (int i = 0; i < IPT; ++i)
            pk[i] = *reinterpret_cast<const uint16_t*>(cbytes + (pk[i] & 0xFFFFu)) + (pk[i] >> 16);
        if (full) {
#pragma unroll
            for (int i = 0; i < IPT; ++i)
                stage[pk[i]] = key[i];
        } else {
#pragma unroll
            for (int i = 0; i < IPT; ++i)
                if (tid * IPT + (uint32_t)i < count)
                    stage[pk[i]] = key[i];
        }
#pragma unroll
        for (uint32_t r = 0; r < L; ++r)
            cnt[r * T + tid] = 0u;
        fence_proxy_async_smem(); // the stage stores come before the bulk copies that read them
        __syncthreads();

        // write-out: one thread per piece sends its 16-byte aligned body with the bulk-copy engine
        // and its up to three slots either side with plain stores
        if (tile_ok != 0u) {
            for (uint32_t p = tid; p < n_pieces; p += T) {
                const uint4 pc = pcs[p];
                const uint32_t g = pc.x, s = pc.y, n = pc.z;
                const uint32_t h = min(n, (4u - (g & 3u)) & 3u);
                const uint32_t nb = (n - h) & ~3u;
                if (nb != 0u)
                    bulk_store(out + g + h, stage + s + h, nb * 4u);
                for (uint32_t i = 0; i < h; ++i)
                    out[g + i] = stage[s + i];
                for (uint32_t i = h + nb; i < n; ++i)
                    out[g + i] = stage[s + i];
            }
            bulk_commit();
        }
    }
    bulk_wait0();
}

// Scratch the kernel needs beyond the per-CTA rows: the control blocks, the tile histograms and
// their 16-byte alignment.
template <typename S>
constexpr uint64_t coop_bulk_fixed_bytes(uint32_t n_tiles)
{
    return sizeof(FusedCtl) + sizeof(CoopHdr) + (uint64_t)n_tiles * S::kHistWords * 4u + 16u;
}

// True when `scratch_bytes` holds the kernel's scratch for at least min(n_tiles, sms) CTAs (the
// dispatcher takes fused_partition_coop_kernel otherwise).
template <typename S>
constexpr bool coop_bulk_fits(uint32_t n_tiles, uint64_t scratch_bytes, int sms)
{
    const uint64_t ctas = n_tiles < (uint32_t)sms ? n_tiles : (uint64_t)sms;
    return scratch_bytes >= coop_bulk_fixed_bytes<S>(n_tiles) + ctas * sizeof(uint32_t) * S::kMaxBins;
}

// Host side: one cooperative launch, as launch_fused_coop; the scratch holds the control block,
// 4 * 2 * LANES bytes per CTA, then (16-byte aligned) the per-tile histograms, and the grid is
// capped by what is left for the per-CTA rows.
template <typename S, typename Cls>
cudaError_t launch_fused_coop_bulk(cudaStream_t stream, Cls cls, const uint32_t* in, uint32_t* out,
                                   uint32_t capacity, uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles,
                                   uint32_t bins, const uint32_t* reserved, uint32_t n_reserved, uint32_t* totals,
                                   unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl,
                                   uint64_t scratch_bytes, uint32_t* status, int sms, InlineFinish fin = {})
{
    auto kernel = fused_partition_coop_bulk_kernel<S, Cls>;
    constexpr uint64_t kRow = sizeof(uint32_t) * S::kMaxBins;
    const uint64_t fixed = coop_bulk_fixed_bytes<S>(n_tiles);
    if (scratch_bytes < fixed + kRow)
        return cudaErrorInvalidValue;
    cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmemBytes);
    if (err != cudaSuccess)
        return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, S::kThreads, S::kSmemBytes);
    if (err != cudaSuccess)
        return err;
    if (per_sm < 1)
        return cudaErrorInvalidConfiguration;
    uint64_t g = (uint64_t)per_sm * (uint64_t)sms;
    g = g < n_tiles ? g : n_tiles;
    const uint64_t cap_ctas = (scratch_bytes - fixed) / kRow;
    g = g < cap_ctas ? g : cap_ctas;
    if (g == 0u)
        return cudaErrorInvalidConfiguration;
    // every CTA owns at most ceil(n_tiles / g) tiles of at most kMaxCount keys: below 2^30 (CoopHdr)
    if (((uint64_t)n_tiles + g - 1u) / g * S::kMaxCount >= (1ull << 30))
        return cudaErrorInvalidConfiguration;
    CoopHdr* hdr = reinterpret_cast<CoopHdr*>(ctl + 1);
    uint32_t* cta_tot = reinterpret_cast<uint32_t*>(hdr + 1);
    uint32_t* tile_hist = reinterpret_cast<uint32_t*>(
        (reinterpret_cast<uintptr_t>(cta_tot + g * S::kMaxBins) + 15u) & ~(uintptr_t)15u);
    err = cudaMemsetAsync(hdr, 0, kCoopHdrResetBytes, stream);
    if (err != cudaSuccess)
        return err;
    FastDiv fd(capacity);
    void* args[] = {&in,      &out,      &cls,        &capacity, &fd,          &pool_slots, &tiles,
                    &n_tiles, &bins,     &reserved,   &n_reserved, &totals,    &port_chunks, &max_k,
                    &ctl,     &hdr,      &cta_tot,    &tile_hist, &status,     &fin};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3((uint32_t)g), dim3(S::kThreads),
                                       args, S::kSmemBytes, stream);
}

} // namespace
} // namespace gf
