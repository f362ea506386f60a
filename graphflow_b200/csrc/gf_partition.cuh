// Partition kernels of the transform-batch hot path (dense bins), templated over the payload
// access policy, the classifier and the updater so that the C ABI (built-in classifiers) and
// the C++ Flow front end (user functors) instantiate the same code.
//
// Reference behaviour restated (paths inside graphFlow's include/graphFlow):
//   classify  flow/Execution.hpp:870-954, graph/ClassifyKernel.hpp:33-93
//   scatter   flow/Execution.hpp:985-1189, graph/ScatterKernel.hpp:174-289 (shared) / :98-173 (direct)
//   plan      graph/DenseBinTable.hpp:39-91 (host) and its device form in fused_finish_kernel
//
// Tile layout inside a CTA: warp w owns the contiguous slice [w*32*IPT, (w+1)*32*IPT) of the tile
// and walks it in IPT rounds of 32 consecutive items, so every global access of a round is one
// coalesced 128-byte (u32) or 512-byte (16 B record) transaction per warp.
#pragma once

#include "gf_device.cuh"

namespace gf {
// Kernels and their helpers have internal linkage: every translation unit that includes this
// header owns its own instantiations, so one kernel is never registered by two modules.
namespace {

// UpdateResult of flow/Concepts.hpp (success / overflow / invalid).
enum : uint32_t { kUpdateSuccess = 0u, kUpdateOverflow = 1u, kUpdateInvalid = 2u };

struct NoUpdate {
    template <typename P>
    GF_D uint32_t operator()(uint32_t, P&, uint64_t /*seed_mixed*/) const
    {
        return kUpdateSuccess;
    }
};

// One u32 column (the kernel-level sweeps' key payload).
struct U32Column {
    using Payload = uint32_t;
    const uint32_t* in;
    uint32_t* out;
    GF_D Payload load(uint64_t slot) const { return ld_stream(in + slot); }
    GF_D void store(uint64_t slot, const Payload& p) const { out[slot] = p; }
    GF_HD static uint64_t key(const Payload& p) { return p; }
};

template <typename Access>
struct KeyClassify {
    KeyClassifier cls;
    GF_D uint32_t operator()(const typename Access::Payload& p) const { return cls(Access::key(p)); }
};

// THREADS threads, IPT items per thread, MINB resident CTAs per SM requested from the register
// allocator (__launch_bounds__ minBlocks).
template <int THREADS, int IPT, int MINB = 1>
struct TileShape {
    static constexpr int kThreads = THREADS;
    static constexpr int kIpt = IPT;
    static constexpr int kMinBlocks = MINB;
    static constexpr int kWarps = THREADS / 32;
    static constexpr int kTile = THREADS * IPT;
    GF_D static uint32_t item(int w, int r, int lane) { return (uint32_t)(w * 32 * IPT + r * 32 + lane); }
};

// An item's bin and its rank inside its warp's slice share one register: bin in bits 0..15
// (0xFFFF = no bin), rank in bits 16..31. Dense partitions therefore take at most 65535 bins.
constexpr uint32_t kNoBin16 = 0xFFFFu;
GF_HD uint32_t bp_bin(uint32_t bp) { return bp & 0xFFFFu; }
GF_HD uint32_t bp_pos(uint32_t bp) { return bp >> 16; }

constexpr uint32_t kNoBin = 0xFFFFFFFFu;
constexpr uint32_t kNoChunk = 0xFFFFFFFFu;

// Block-wide exclusive scan of n <= 65536 u32 values held in shared memory (in-place allowed).
// `warp_tmp` needs kWarps + 1 words. Returns the total to every thread.
template <int THREADS>
GF_D uint32_t block_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* warp_tmp)
{
    constexpr int W = THREADS / 32;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint32_t per = (n + THREADS - 1) / THREADS;
    const uint32_t lo = min(n, (uint32_t)tid * per), hi = min(n, lo + per);
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; ++i)
        sum += in[i];
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o)
            incl += v;
    }
    if (lane == 31)
        warp_tmp[w] = incl;
    __syncthreads();
    if (tid == 0) {
        uint32_t run = 0;
        for (int i = 0; i < W; ++i) {
            uint32_t c = warp_tmp[i];
            warp_tmp[i] = run;
            run += c;
        }
        warp_tmp[W] = run;
    }
    __syncthreads();
    uint32_t run = warp_tmp[w] + incl - sum;
    for (uint32_t i = lo; i < hi; ++i) {
        uint32_t c = in[i];
        out[i] = run;
        run += c;
    }
    uint32_t total = warp_tmp[W];
    __syncthreads();
    return total;
}

// Stable in-tile ranking. bp[r] holds the bin of item (w, r, lane) in its low half (kNoBin16 for
// none). On return its high half holds the item's rank among the items of its bin inside its
// warp's slice, and warp_cnt[w*B + b] holds the number of items of bin b in warp w's slice.
// The lanes that share an item's bin: match.any, whose cost grows with the number of distinct
// values in the warp, except for 17 to 64 bins: one ballot for "has a bin" and one per bin bit
// (7 ballots at 64 bins, about a third of match.any's cost there; at 16 bins and fewer match.any
// measured cheaper).
template <typename Shape>
GF_D void warp_rank(uint32_t (&bp)[Shape::kIpt], uint32_t* warp_cnt, uint32_t B)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t* cnt = warp_cnt + (size_t)w * B;
    for (uint32_t b = lane; b < B; b += 32)
        cnt[b] = 0u;
    __syncwarp();
    const uint32_t lt = lanemask_lt();
    // bits of a bin, or -1: match.any
    const int nbits = B > 16u && B <= 64u ? 32 - __clz((int)(B - 1u)) : -1;
#pragma unroll
    for (int r = 0; r < Shape::kIpt; ++r) {
        const uint32_t bin = bp_bin(bp[r]);
        uint32_t peers;
        if (nbits >= 0) {
            const uint32_t valid = __ballot_sync(0xFFFFFFFFu, bin != kNoBin16);
            peers = bin != kNoBin16 ? valid : ~valid;
            for (int k = 0; k < nbits; ++k) {
                const uint32_t bit = (bin >> k) & 1u;
                const uint32_t set = __ballot_sync(0xFFFFFFFFu, bit != 0u);
                peers &= bit != 0u ? set : ~set;
            }
        } else {
            peers = __match_any_sync(0xFFFFFFFFu, bin);
        }
        uint32_t base = 0;
        if (bin != kNoBin16)
            base = cnt[bin];
        __syncwarp();
        if (bin != kNoBin16) {
            bp[r] = bin | ((base + __popc(peers & lt)) << 16);
            if (lane == 31 - __clz(peers))
                cnt[bin] = base + __popc(peers);
        }
        __syncwarp();
    }
}

// Per-bin warp offsets (exclusive over warps, in place) and tile totals.
template <typename Shape>
GF_D void warp_offsets(uint32_t* warp_cnt, uint32_t* bin_tot, uint32_t B)
{
    for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < Shape::kWarps; ++w) {
            uint32_t c = warp_cnt[(size_t)w * B + b];
            warp_cnt[(size_t)w * B + b] = run;
            run += c;
        }
        bin_tot[b] = run;
    }
}

// ---------------------------------------------------------------------------------------------
// Classify: flow/Execution.hpp:870-954. Per tile: classify every payload, store its bin, count
// bins in shared memory with warp-aggregated atomics, then one device atomic per (tile, bin).
// counts[B] is the status slot.
// ---------------------------------------------------------------------------------------------
template <typename Shape, typename Access, typename Classify>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) classify_kernel(Access acc, Classify classify, uint32_t capacity,
                                                                   uint64_t pool_slots, const gf_tile* tiles,
                                                                   uint32_t n_tiles, uint32_t B, uint32_t* bin_ids,
                                                                   uint32_t* counts, uint32_t* status)
{
    extern __shared__ uint32_t smem[];
    uint32_t* hist = smem; // [B]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const gf_tile tile = tiles[t];
        const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
        const bool tile_ok = tile.count <= (uint32_t)Shape::kTile && base + tile.count <= pool_slots &&
                             tile.tile_offset + tile.count <= capacity;
        for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads)
            hist[b] = 0u;
        __syncthreads();
        if (!tile_ok) {
            if (threadIdx.x == 0)
                set_status(status, GF_INVALID);
        } else {
            typename Access::Payload p[Shape::kIpt];
#pragma unroll
            for (int r = 0; r < Shape::kIpt; ++r) {
                const uint32_t i = Shape::item(w, r, lane);
                if (i < tile.count)
                    p[r] = acc.load(base + i);
            }
#pragma unroll
            for (int r = 0; r < Shape::kIpt; ++r) {
                const uint32_t i = Shape::item(w, r, lane);
                uint32_t bin = kNoBin;
                if (i < tile.count) {
                    bin = classify(p[r]);
                    if (bin >= B) {
                        counts[B] = 1u;
                        set_status(status, GF_INVALID);
                        bin = kNoBin;
                    } else {
                        bin_ids[base + i] = bin;
                    }
                }
                const uint32_t peers = __match_any_sync(0xFFFFFFFFu, bin);
                if (bin != kNoBin && lane == 31 - __clz(peers))
                    atomicAdd(&hist[bin], (uint32_t)__popc(peers));
            }
        }
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads)
            if (hist[b] != 0u)
                atomicAdd(&counts[b], hist[b]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Scatter (SharedStaging): flow/Execution.hpp:1096-1187. Per tile: recount from the stored bins,
// reserve one range per bin with a device atomic on next[bin], rank inside the tile (stable),
// apply the updater, stage the tile in shared memory in bin order and write it out coalesced:
// out slot = table[B + table[bin] + j / C] * C + j % C.
// ---------------------------------------------------------------------------------------------
template <typename Shape, typename Access, typename Update>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) scatter_kernel(Access acc, Update update, uint64_t seed_mixed,
                                                                  uint32_t capacity, FastDiv fdc, uint64_t pool_slots,
                                                                  const gf_tile* tiles, uint32_t n_tiles, uint32_t B,
                                                                  const uint32_t* bin_ids, const uint32_t* table,
                                                                  uint32_t* next, uint32_t* counts, uint32_t* status)
{
    using P = typename Access::Payload;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* stage = reinterpret_cast<P*>(smem_raw);
    uint32_t* stage_bin = reinterpret_cast<uint32_t*>(stage + Shape::kTile);
    uint32_t* warp_cnt = stage_bin + Shape::kTile;            // [W][B]
    uint32_t* bin_tot = warp_cnt + (size_t)Shape::kWarps * B; // [B]
    uint32_t* bin_excl = bin_tot + B;                         // [B]
    uint32_t* gbase = bin_excl + B;                           // [B]
    uint32_t* scan_tmp = gbase + B;                           // [W+1]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const gf_tile tile = tiles[t];
        const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
        const bool tile_ok = tile.count <= (uint32_t)Shape::kTile && base + tile.count <= pool_slots &&
                             tile.tile_offset + tile.count <= capacity;
        uint32_t bp[Shape::kIpt];
        P p[Shape::kIpt];
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            bp[r] = kNoBin16;
            if (tile_ok && i < tile.count) {
                const uint32_t b = __ldg(bin_ids + base + i);
                p[r] = acc.load(base + i);
                if (b >= B) {
                    counts[B] = 1u;
                    set_status(status, GF_INVALID);
                } else {
                    bp[r] = b;
                }
            }
        }
        if (!tile_ok && threadIdx.x == 0)
            set_status(status, GF_INVALID);
        warp_rank<Shape>(bp, warp_cnt, B);
        __syncthreads();
        warp_offsets<Shape>(warp_cnt, bin_tot, B);
        __syncthreads();
        const uint32_t n_valid = block_exclusive_scan<Shape::kThreads>(bin_tot, bin_excl, B, scan_tmp);
        for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads)
            if (bin_tot[b] != 0u)
                gbase[b] = atomicAdd(&next[b], bin_tot[b]) - bin_excl[b];
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t b = bp_bin(bp[r]);
            if (b != kNoBin16) {
                const uint32_t q = bin_excl[b] + warp_cnt[(size_t)w * B + b] + bp_pos(bp[r]);
                const uint32_t res = update(b, p[r], seed_mixed);
                if (res != kUpdateSuccess) {
                    counts[B] = 1u;
                    set_status(status, res == kUpdateOverflow ? GF_OVERFLOW : GF_INVALID);
                }
                stage[q] = p[r];
                stage_bin[q] = b;
            }
        }
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < n_valid; q += Shape::kThreads) {
            const uint32_t b = stage_bin[q];
            const uint32_t j = gbase[b] + q;
            const uint32_t k = fdc.div(j);
            const uint32_t chunk = __ldg(table + B + __ldg(table + b) + k);
            const uint64_t slot = (uint64_t)chunk * capacity + (j - k * capacity);
            if (slot < pool_slots)
                acc.store(slot, stage[q]);
            else
                set_status(status, GF_OVERFLOW);
        }
        __syncthreads();
    }
}

// Scatter (Direct): flow/Execution.hpp:1034-1095, one device atomic per particle.
template <typename Shape, typename Access, typename Update>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) scatter_direct_kernel(Access acc, Update update,
                                                                         uint64_t seed_mixed, uint32_t capacity,
                                                                         FastDiv fdc, uint64_t pool_slots,
                                                                         const gf_tile* tiles, uint32_t n_tiles,
                                                                         uint32_t B, const uint32_t* bin_ids,
                                                                         const uint32_t* table, uint32_t* next,
                                                                         uint32_t* counts, uint32_t* status)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const gf_tile tile = tiles[t];
        const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
        if (tile.count > (uint32_t)Shape::kTile || base + tile.count > pool_slots ||
            tile.tile_offset + tile.count > capacity) {
            if (threadIdx.x == 0)
                set_status(status, GF_INVALID);
            continue;
        }
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            if (i >= tile.count)
                continue;
            const uint32_t b = __ldg(bin_ids + base + i);
            if (b >= B) {
                counts[B] = 1u;
                set_status(status, GF_INVALID);
                continue;
            }
            const uint32_t j = atomicAdd(&next[b], 1u);
            const uint32_t k = fdc.div(j);
            const uint32_t chunk = __ldg(table + B + __ldg(table + b) + k);
            const uint64_t slot = (uint64_t)chunk * capacity + (j - k * capacity);
            typename Access::Payload p = acc.load(base + i);
            const uint32_t res = update(b, p, seed_mixed);
            if (res != kUpdateSuccess) {
                counts[B] = 1u;
                set_status(status, res == kUpdateOverflow ? GF_OVERFLOW : GF_INVALID);
            }
            if (slot < pool_slots)
                acc.store(slot, p);
            else
                set_status(status, GF_OVERFLOW);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Fused single-pass classify -> scan -> scatter.
//
// Scratch: a control block {tile counter, allocation cursor} that the host zeroes per launch,
// followed by one 64-bit look-back descriptor per (tile, bin):
//   bits 63..34 epoch, 33..32 flag (1 = tile aggregate, 2 = inclusive prefix), 31..0 value.
// Descriptors of older launches carry an older epoch and read as "not ready", so the array
// needs no clearing. Tiles take their index from the counter in launch order, so every tile a
// CTA waits on belongs to a CTA that is already running; every wait is still bounded.
// ---------------------------------------------------------------------------------------------
struct FusedCtl {
    uint32_t tile_counter; // reset by the host before every launch
    uint32_t alloc_cursor; // reset by the host before every launch
    uint32_t done;         // reset by the host before every launch
    uint32_t epoch;        // persistent: epoch of the last completed launch (0 = none yet)
    uint32_t pad[12];
};
constexpr uint32_t kFusedCtlResetBytes = 3u * sizeof(uint32_t);

GF_HD uint32_t next_epoch(uint32_t e) { return (e % 0x3FFFFFFFu) + 1u; } // 30-bit, never 0

GF_HD unsigned long long make_desc(uint32_t epoch, uint32_t flag, uint32_t value)
{
    return ((unsigned long long)((epoch << 2) | flag) << 32) | value;
}

constexpr uint32_t kClaimed = 0xFFFFFFFEu;

// Back-off step of a bounded wait: false when the wait must give up (poll budget spent, or the
// batch's status word already reports a failure).
GF_D bool poll_again(uint32_t& polls, const uint32_t* status)
{
    if (++polls >= g_spin_limit)
        return false;
    if ((polls & 255u) == 0u && ld_relaxed_u32(status) != 0u)
        return false;
    __nanosleep(polls < 64u ? 20u : 40u);
    return true;
}

// Chunk k of a port's output range, taken on first touch: whichever tile touches it first claims
// the slot with a CAS (tagging it with this launch's epoch), takes the next reserved chunk and
// publishes it; later touchers read it, waiting (bounded) only while a claim is in flight.
// Because any toucher may claim, no tile waits for the look-back of the tile that owns the
// chunk's first position.
GF_D uint32_t claim_chunk(unsigned long long* slot, uint32_t epoch, uint32_t* alloc_cursor, const uint32_t* reserved,
                          uint32_t n_reserved, uint32_t* status)
{
    const unsigned long long tag = (unsigned long long)epoch << 32;
    unsigned long long v = ld_relaxed_u64(slot);
    if ((uint32_t)(v >> 32) != epoch) {
        const unsigned long long old = atomicCAS(slot, v, tag | kClaimed);
        if (old == v) {
            const uint32_t idx = atomicAdd(alloc_cursor, 1u);
            uint32_t chunk = kNoChunk;
            if (idx < n_reserved)
                chunk = __ldg(reserved + idx);
            else
                set_status(status, GF_OVERFLOW);
            st_relaxed_u64(slot, tag | chunk);
            return chunk;
        }
        v = old;
    }
    uint32_t polls = 0;
    while ((uint32_t)(v >> 32) != epoch || (uint32_t)v == kClaimed) {
        if (!poll_again(polls, status)) {
            set_status(status, GF_ERR_TIMEOUT);
            return kNoChunk;
        }
        v = ld_relaxed_u64(slot);
    }
    return (uint32_t)v;
}

// Block-wide decoupled look-back over the per-(tile, bin) descriptors of tile t > 0.
// Pass p covers bins [p*P, p*P + P) with P = min(B, THREADS); each of the W = THREADS / P thread
// groups reads one predecessor, so one round reads a window of W predecessors for P bins at once.
// Per bin, the window is reduced up to the nearest inclusive prefix; bins without one move the
// window further back. On return acc[b] holds bin b's exclusive prefix over tiles 0..t-1.
template <int THREADS>
GF_D void block_lookback(const unsigned long long* desc, uint32_t t, uint32_t B, uint32_t epoch_hi, uint32_t* acc,
                         uint32_t* done, uint32_t* lb_flag, uint32_t* lb_val, uint32_t* status)
{
    const uint32_t P = B < (uint32_t)THREADS ? B : (uint32_t)THREADS;
    const uint32_t W = (uint32_t)THREADS / P;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane_bin = tid % P, woff = tid / P;
    for (uint32_t pass = 0; pass < B; pass += P) {
        const uint32_t b = pass + lane_bin;
        const bool owner = tid < P && b < B;
        if (owner) {
            acc[b] = 0u;
            done[b] = 0u;
        }
        __syncthreads();
        int64_t pred_base = (int64_t)t - 1;
        for (;;) {
            uint32_t flag = 2u, val = 0u;
            if (woff < W && b < B && done[b] == 0u) {
                const int64_t pred = pred_base - (int64_t)woff;
                if (pred >= 0) {
                    const unsigned long long* d = desc + (size_t)pred * B + b;
                    unsigned long long v = ld_relaxed_u64(d);
                    uint32_t polls = 0;
                    bool ok = true;
                    while ((uint32_t)(v >> 34) != epoch_hi || ((v >> 32) & 3u) == 0u) {
                        if (!poll_again(polls, status)) {
                            ok = false;
                            break;
                        }
                        v = ld_relaxed_u64(d);
                    }
                    if (ok) {
                        flag = (uint32_t)(v >> 32) & 3u;
                        val = (uint32_t)v;
                    } else {
                        set_status(status, GF_ERR_TIMEOUT);
                    }
                }
            }
            lb_flag[tid] = flag;
            lb_val[tid] = val;
            __syncthreads();
            if (owner && done[b] == 0u) {
                uint32_t a = acc[b];
                for (uint32_t j = 0; j < W; ++j) {
                    a += lb_val[j * P + lane_bin];
                    if (lb_flag[j * P + lane_bin] == 2u) {
                        done[b] = 1u;
                        break;
                    }
                }
                acc[b] = a;
            }
            if (__syncthreads_and(!owner || done[b] != 0u))
                break;
            pred_base -= (int64_t)W;
        }
    }
}

// Optional in-kernel finish of a fused launch: when `table` is set, the last CTA of the launch
// builds the chunk table, the output descriptors and the output count itself (what
// fused_finish_kernel does), so a caller that would launch the finish right after saves a launch.
struct InlineFinish {
    uint32_t* table = nullptr;
    gf_out_desc* descs = nullptr;
    uint32_t desc_cap = 0u;
    uint32_t* num_out = nullptr;
    // Host-polled completion (per-tile kernel only): a record in mapped host memory,
    // [0] sequence, [1] status, [2] output count, [3, 3 + B) totals, then the descriptors. The
    // finishing CTA fills it, resets the launch counters for the next launch and writes `done_seq`
    // last, so a host that sees the sequence reads a complete record without a copy or an event.
    uint32_t* done_rec = nullptr;
    uint32_t done_seq = 0u;
};

// The finishing CTA of a launch with a host-polled completion record (see InlineFinish).
GF_D void publish_done(const InlineFinish& fin, FusedCtl* ctl, const uint32_t* totals, uint32_t B,
                       uint32_t* status)
{
    __syncthreads(); // the finish's table, descriptors and output count are written
    uint32_t* rec = fin.done_rec;
    const uint32_t r = ld_relaxed_u32(fin.num_out);
    const uint32_t nd = 3u * (r < fin.desc_cap ? r : fin.desc_cap);
    const uint32_t* d = reinterpret_cast<const uint32_t*>(fin.descs);
    for (uint32_t i = threadIdx.x; i < B; i += blockDim.x)
        rec[3u + i] = ld_relaxed_u32(totals + i);
    for (uint32_t i = threadIdx.x; i < nd; i += blockDim.x)
        rec[3u + B + i] = ld_relaxed_u32(d + i);
    if (threadIdx.x == 0) {
        // every CTA has counted itself: the counters are free for the next launch
        ctl->tile_counter = 0u;
        ctl->alloc_cursor = 0u;
        ctl->done = 0u;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        rec[1] = ld_relaxed_u32(status);
        rec[2] = r;
        *status = 0u; // read into the record: the word is clean for the next launch
        __threadfence_system();
        *reinterpret_cast<volatile uint32_t*>(rec) = fin.done_seq;
    }
}

// Device form of planDenseBins + buildDenseTable + the output-descriptor loop
// (DenseBinTable.hpp:39-91, Execution.hpp:2558-2581) for a fused launch, by one CTA of THREADS
// threads: bins in segments of `seg` (nck and base hold `seg` words each, tmp THREADS / 32 + 1),
// one thread per output chunk of a segment. Totals and chunk claims are read from L2, so the last
// CTA of the fused launch itself can run it after the launch's other CTAs retired.
template <int THREADS>
GF_D void finish_plan(const uint32_t* totals, const unsigned long long* port_chunks, uint32_t B, uint32_t capacity,
                      FastDiv fdc, uint32_t max_k, uint32_t epoch, uint32_t* table, gf_out_desc* descs,
                      uint32_t desc_cap, uint32_t* num_out, uint32_t* status, uint32_t* nck, uint32_t* base,
                      uint32_t seg_words, uint32_t* tmp)
{
    uint32_t carry = 0;
    for (uint32_t seg = 0; seg < B; seg += seg_words) {
        const uint32_t n = min(seg_words, B - seg);
        for (uint32_t i = threadIdx.x; i < n; i += THREADS) {
            const uint32_t tot = ld_relaxed_u32(totals + seg + i);
            nck[i] = fdc.div(tot) + (fdc.mod(tot) != 0u ? 1u : 0u);
        }
        __syncthreads();
        const uint32_t sum = block_exclusive_scan<THREADS>(nck, base, n, tmp);
        for (uint32_t i = threadIdx.x; i < n; i += THREADS)
            table[seg + i] = carry + base[i];
        // one thread per output chunk of the segment (a port may own most of them)
        for (uint32_t g = threadIdx.x; g < sum; g += THREADS) {
            uint32_t lo = 0, hi = n - 1u; // the last port of the segment whose chunks start at or before g
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1u) >> 1;
                if (base[mid] <= g)
                    lo = mid;
                else
                    hi = mid - 1u;
            }
            const uint32_t b = seg + lo, k = g - base[lo], f = carry + g;
            if (f >= desc_cap || k >= max_k) {
                set_status(status, GF_OVERFLOW);
                continue;
            }
            const unsigned long long v = ld_relaxed_u64(port_chunks + (size_t)b * max_k + k);
            const uint32_t chunk = (uint32_t)(v >> 32) == epoch ? (uint32_t)v : kNoChunk;
            if (chunk == kNoChunk)
                set_status(status, GF_INVALID);
            table[B + f] = chunk;
            descs[f].chunk_index = chunk;
            descs[f].fill = min(capacity, ld_relaxed_u32(totals + b) - k * capacity);
            descs[f].bin = b;
        }
        carry += sum;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *num_out = carry;
}

// Work of the finishing CTA after an inline finish (all of its threads call it once the table,
// descriptors and output count are written): none by default.
struct NoPost {
    static constexpr bool kActive = false;
    GF_D void operator()(const InlineFinish&, uint32_t*) const {}
};

template <typename Shape, typename Access, typename Classify, typename Update, typename Post = NoPost>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) fused_partition_kernel(
    Access acc, Classify classify, Update update, uint64_t seed_mixed, uint32_t capacity, FastDiv fdc,
    uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t B, const uint32_t* reserved,
    uint32_t n_reserved, uint32_t* totals, unsigned long long* port_chunks, uint32_t max_k, FusedCtl* ctl,
    unsigned long long* desc, uint32_t* status, InlineFinish fin, Post post)
{
    using P = typename Access::Payload;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* stage = reinterpret_cast<P*>(smem_raw);
    uint32_t* stage_bin = reinterpret_cast<uint32_t*>(stage + Shape::kTile);
    uint32_t* warp_cnt = stage_bin + Shape::kTile;            // [W][B]
    uint32_t* bin_tot = warp_cnt + (size_t)Shape::kWarps * B; // [B]
    uint32_t* bin_excl = bin_tot + B;                         // [B]
    uint32_t* gbase = bin_excl + B;                           // [B]
    uint32_t* k0 = gbase + B;                                 // [B]
    uint32_t* chunk_lo = k0 + B;                              // [B]
    uint32_t* chunk_hi = chunk_lo + B;                        // [B]
    uint32_t* lb_flag = chunk_hi + B;                         // [THREADS]
    uint32_t* lb_val = lb_flag + Shape::kThreads;             // [THREADS]
    uint32_t* scan_tmp = lb_val + Shape::kThreads;            // [W+1]
    uint32_t* s_tile = scan_tmp + Shape::kWarps + 1;          // [6]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    // The launch epoch is the successor of the last completed launch's epoch; the last CTA to
    // finish publishes it, so CUDA-graph replays of this launch get a fresh epoch each time. One
    // thread reads the tile descriptor (the list may sit in mapped host memory).
    if (threadIdx.x == 0) {
        const uint32_t tt = atomicAdd(&ctl->tile_counter, 1u);
        s_tile[0] = tt;
        s_tile[1] = next_epoch(ld_relaxed_u32(&ctl->epoch));
        if (tt < n_tiles) {
            const gf_tile tl = tiles[tt];
            s_tile[3] = tl.chunk_index;
            s_tile[4] = tl.tile_offset;
            s_tile[5] = tl.count;
        }
    }
    __syncthreads();
    const uint32_t t = s_tile[0];
    const uint32_t epoch = s_tile[1];
    const uint32_t epoch_hi = epoch;
    // retire this CTA; with an inline finish, the last CTA then builds the table and descriptors
    // (its stage area and look-back words are free by then)
    auto retire = [&]() {
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const bool last = atomicAdd(&ctl->done, 1u) + 1u == gridDim.x;
            if (last)
                atomicExch(&ctl->epoch, epoch);
            s_tile[2] = last ? 1u : 0u;
        }
        if (fin.table == nullptr)
            return;
        __syncthreads();
        if (s_tile[2] == 0u)
            return;
        __threadfence(); // every other CTA's totals and chunk claims were published before its arrival
        constexpr uint32_t kSeg = (uint32_t)(sizeof(P) * Shape::kTile / 8u);
        uint32_t* scratch = reinterpret_cast<uint32_t*>(smem_raw);
        finish_plan<Shape::kThreads>(totals, port_chunks, B, capacity, fdc, max_k, epoch, fin.table, fin.descs,
                                     fin.desc_cap, fin.num_out, status, scratch, scratch + kSeg, kSeg, lb_flag);
        if (fin.done_rec != nullptr)
            publish_done(fin, ctl, totals, B, status);
        if constexpr (Post::kActive) {
            __syncthreads();
            post(fin, status);
        }
    };
    if (t >= n_tiles) {
        retire();
        return;
    }

    const gf_tile tile{s_tile[3], s_tile[4], s_tile[5]};
    const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
    const bool tile_ok = tile.count <= (uint32_t)Shape::kTile && base + tile.count <= pool_slots &&
                         tile.tile_offset + tile.count <= capacity;
    if (!tile_ok && threadIdx.x == 0)
        set_status(status, GF_INVALID);

    // 1. load and classify
    uint32_t bp[Shape::kIpt];
    P p[Shape::kIpt];
#pragma unroll
    for (int r = 0; r < Shape::kIpt; ++r) {
        const uint32_t i = Shape::item(w, r, lane);
        bp[r] = kNoBin16;
        if (tile_ok && i < tile.count)
            p[r] = acc.load(base + i);
    }
#pragma unroll
    for (int r = 0; r < Shape::kIpt; ++r) {
        const uint32_t i = Shape::item(w, r, lane);
        if (tile_ok && i < tile.count) {
            const uint32_t b = classify(p[r]);
            if (b >= B)
                set_status(status, GF_INVALID);
            else
                bp[r] = b;
        }
    }
    // 2. stable rank inside the tile, per-bin tile totals
    warp_rank<Shape>(bp, warp_cnt, B);
    __syncthreads();
    warp_offsets<Shape>(warp_cnt, bin_tot, B);
    __syncthreads();

    // 3. publish the tile aggregate, then look back for the exclusive prefix of every bin
    unsigned long long* my_desc = desc + (size_t)t * B;
    for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads)
        st_relaxed_u64(my_desc + b, make_desc(epoch_hi, t == 0 ? 2u : 1u, bin_tot[b]));
    const uint32_t n_valid = block_exclusive_scan<Shape::kThreads>(bin_tot, bin_excl, B, scan_tmp);

    // 4. apply the updater and stage the tile in bin order (tile-local positions only)
#pragma unroll
    for (int r = 0; r < Shape::kIpt; ++r) {
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

    // 5. block-wide windowed look-back: every pass covers P bins x W predecessors with all
    //    threads loading in parallel; excl[b] accumulates in gbase[b], done flags in chunk_lo[b]
    if (t != 0u)
        block_lookback<Shape::kThreads>(desc, t, B, epoch_hi, gbase, chunk_lo, lb_flag, lb_val, status);
    else
        for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads)
            gbase[b] = 0u;
    __syncthreads();

    // 6. publish the inclusive prefixes, then take this range's output chunks by first-touch claim
    for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads) {
        const uint32_t excl = gbase[b], tot = bin_tot[b];
        if (t != 0u)
            st_relaxed_u64(my_desc + b, make_desc(epoch_hi, 2u, excl + tot));
        if (t + 1u == n_tiles)
            totals[b] = excl + tot;
        gbase[b] = excl - bin_excl[b];
        uint32_t lo = kNoChunk, hi = kNoChunk;
        if (tot != 0u) {
            const uint32_t ka = fdc.div(excl), kb = fdc.div(excl + tot - 1u);
            k0[b] = ka;
            if (kb >= max_k) {
                set_status(status, GF_OVERFLOW);
            } else {
                lo = claim_chunk(port_chunks + (size_t)b * max_k + ka, epoch, &ctl->alloc_cursor, reserved,
                                 n_reserved, status);
                if (kb != ka)
                    hi = claim_chunk(port_chunks + (size_t)b * max_k + kb, epoch, &ctl->alloc_cursor, reserved,
                                     n_reserved, status);
            }
        }
        chunk_lo[b] = lo;
        chunk_hi[b] = hi;
    }
    if (threadIdx.x == 0)
        s_tile[2] = ld_relaxed_u32(status);
    __syncthreads();
    if (s_tile[2] != 0u) {
        retire(); // the batch failed somewhere: write nothing, the host discards it
        return;
    }

    // 7. coalesced write-out
    for (uint32_t q = threadIdx.x; q < n_valid; q += Shape::kThreads) {
        const uint32_t b = stage_bin[q];
        const uint32_t j = gbase[b] + q;
        const uint32_t k = fdc.div(j);
        const uint32_t chunk = k == k0[b] ? chunk_lo[b] : chunk_hi[b];
        if (chunk == kNoChunk)
            continue;
        const uint64_t slot = (uint64_t)chunk * capacity + (j - k * capacity);
        if (slot < pool_slots)
            acc.store(slot, stage[q]);
        else
            set_status(status, GF_OVERFLOW);
    }
    retire();
}

// One partition batch of a multi-batch fused launch (several nodes' ready batches in one grid):
// its tiles in the launch's tile list, the node (member) whose classifier and updater it uses,
// its output-chunk reservation, and its own outputs and scratch. The host zeroes `counters`
// (allocation cursor, retired tiles) before every launch.
struct MultiBatch {
    uint32_t tile_begin;
    uint32_t n_tiles;
    uint32_t member;
    uint32_t n_reserved;
    const uint32_t* reserved;
    uint32_t* totals;                // [B]
    unsigned long long* port_chunks; // [B * max_k]
    unsigned long long* desc;        // [n_tiles * B] look-back descriptors
    uint32_t* counters;              // [2]
    uint32_t* table;                 // [B + desc_cap]
    gf_out_desc* descs;              // [desc_cap]
    uint32_t desc_cap;
    uint32_t* num_out;
};

// Multi-batch form of fused_partition_kernel: one CTA per tile of the concatenated tile list
// (`tile_batch[t]` = the tile's batch). A tile looks back only over the predecessors of its own
// batch, which claimed their tiles earlier from the launch-wide counter, so every wait ends. The
// batch's last tile to retire builds that batch's chunk table and descriptors and resets the
// batch's counters; the launch's last CTA publishes the epoch and resets the launch counters. The
// batches of one launch share the epoch, so their descriptor and chunk-claim words from earlier
// launches read as stale. With `done_rec` (mapped host memory: [0] sequence, [1] status), the last
// of the `live_batches` batches to finish copies the status word there and then writes `done_seq`,
// so the host polls one word instead of an event.
template <typename Shape, typename Access, typename Classify, typename Update>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) fused_partition_multi_kernel(
    Access acc, const Classify* classify_of, const Update* update_of, uint64_t seed_mixed, uint32_t capacity,
    FastDiv fdc, uint64_t pool_slots, const gf_tile* tiles, const uint32_t* tile_batch, uint32_t n_tiles, uint32_t B,
    const MultiBatch* batches, uint32_t n_batches, uint32_t max_k, FusedCtl* ctl, uint32_t* status,
    uint32_t* done_rec, uint32_t done_seq, uint32_t live_batches)
{
    using P = typename Access::Payload;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* stage = reinterpret_cast<P*>(smem_raw);
    uint32_t* stage_bin = reinterpret_cast<uint32_t*>(stage + Shape::kTile);
    uint32_t* warp_cnt = stage_bin + Shape::kTile;            // [W][B]
    uint32_t* bin_tot = warp_cnt + (size_t)Shape::kWarps * B; // [B]
    uint32_t* bin_excl = bin_tot + B;                         // [B]
    uint32_t* gbase = bin_excl + B;                           // [B]
    uint32_t* k0 = gbase + B;                                 // [B]
    uint32_t* chunk_lo = k0 + B;                              // [B]
    uint32_t* chunk_hi = chunk_lo + B;                        // [B]
    uint32_t* lb_flag = chunk_hi + B;                         // [THREADS]
    uint32_t* lb_val = lb_flag + Shape::kThreads;             // [THREADS]
    uint32_t* scan_tmp = lb_val + Shape::kThreads;            // [W+1]
    uint32_t* s_tile = scan_tmp + Shape::kWarps + 1;          // [3]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    // one thread reads the tile's batch record and descriptor (they sit in mapped host memory) into
    // the stage area, which is free until step 4
    uint32_t* s_rec = reinterpret_cast<uint32_t*>(smem_raw);
    constexpr uint32_t kRecWords = (uint32_t)(sizeof(MultiBatch) / 4u);
    if (threadIdx.x == 0) {
        const uint32_t g0 = atomicAdd(&ctl->tile_counter, 1u);
        s_tile[0] = g0;
        s_tile[1] = next_epoch(ld_relaxed_u32(&ctl->epoch));
        const uint32_t b0 = g0 < n_tiles ? tile_batch[g0] : 0u;
        s_tile[2] = b0;
        if (g0 < n_tiles && b0 < n_batches) {
            const uint2* src = reinterpret_cast<const uint2*>(batches + b0);
            uint2* dst = reinterpret_cast<uint2*>(s_rec);
            for (uint32_t i = 0; i < kRecWords / 2u; ++i)
                dst[i] = src[i];
            const gf_tile tl = tiles[g0];
            s_rec[kRecWords] = tl.chunk_index;
            s_rec[kRecWords + 1u] = tl.tile_offset;
            s_rec[kRecWords + 2u] = tl.count;
        }
    }
    __syncthreads();
    const uint32_t gt = s_tile[0];
    const uint32_t epoch = s_tile[1];
    const uint32_t bi = s_tile[2];
    const bool in_range = gt < n_tiles && bi < n_batches;
    if (gt < n_tiles && !in_range && threadIdx.x == 0)
        set_status(status, GF_INVALID);
    const MultiBatch mb = in_range ? *reinterpret_cast<const MultiBatch*>(s_rec) : MultiBatch{};
    const gf_tile tile{s_rec[kRecWords], s_rec[kRecWords + 1u], s_rec[kRecWords + 2u]};
    const uint32_t t = gt - mb.tile_begin; // the tile's index inside its batch
    const bool batch_ok = in_range && gt >= mb.tile_begin && t < mb.n_tiles;
    if (in_range && !batch_ok && threadIdx.x == 0)
        set_status(status, GF_INVALID);
    __syncthreads(); // the record is in registers: the stage area is free again

    // retire: the batch's last tile builds the batch's table and descriptors; the launch's last
    // CTA publishes the epoch
    auto retire = [&]() {
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            uint32_t last_of_batch = 0u;
            if (batch_ok)
                last_of_batch = atomicAdd(mb.counters + 1, 1u) + 1u == mb.n_tiles ? 1u : 0u;
            if (atomicAdd(&ctl->done, 1u) + 1u == gridDim.x) {
                // every CTA has counted itself: the launch counters are free for the next launch
                atomicExch(&ctl->epoch, epoch);
                ctl->tile_counter = 0u;
                ctl->done = 0u;
            }
            s_tile[2] = last_of_batch;
        }
        __syncthreads();
        if (s_tile[2] == 0u)
            return;
        __threadfence(); // the batch's other tiles published their totals and claims before arriving
        constexpr uint32_t kSeg = (uint32_t)(sizeof(P) * Shape::kTile / 8u);
        uint32_t* scratch = reinterpret_cast<uint32_t*>(smem_raw);
        finish_plan<Shape::kThreads>(mb.totals, mb.port_chunks, B, capacity, fdc, max_k, epoch, mb.table, mb.descs,
                                     mb.desc_cap, mb.num_out, status, scratch, scratch + kSeg, kSeg, lb_flag);
        __syncthreads();
        if (threadIdx.x == 0) {
            mb.counters[0] = 0u; // the batch's claims and tiles are all counted
            mb.counters[1] = 0u;
            if (done_rec != nullptr) {
                __threadfence_system(); // this batch's descriptors and output count reach the host first
                if (atomicAdd(&ctl->alloc_cursor, 1u) + 1u == live_batches) {
                    ctl->alloc_cursor = 0u;
                    __threadfence(); // every other batch's finish came before its count
                    done_rec[1] = ld_relaxed_u32(status);
                    *status = 0u;
                    __threadfence_system();
                    *reinterpret_cast<volatile uint32_t*>(done_rec) = done_seq;
                }
            }
        }
    };
    if (!batch_ok) {
        retire();
        return;
    }
    const Classify classify = classify_of[mb.member];
    const Update update = update_of[mb.member];

    const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
    const bool tile_ok = tile.count <= (uint32_t)Shape::kTile && base + tile.count <= pool_slots &&
                         tile.tile_offset + tile.count <= capacity;
    if (!tile_ok && threadIdx.x == 0)
        set_status(status, GF_INVALID);

    // 1. load and classify
    uint32_t bp[Shape::kIpt];
    P p[Shape::kIpt];
#pragma unroll
    for (int r = 0; r < Shape::kIpt; ++r) {
        const uint32_t i = Shape::item(w, r, lane);
        bp[r] = kNoBin16;
        if (tile_ok && i < tile.count)
            p[r] = acc.load(base + i);
    }
#pragma unroll
    for (int r = 0; r < Shape::kIpt; ++r) {
        const uint32_t i = Shape::item(w, r, lane);
        if (tile_ok && i < tile.count) {
            const uint32_t b = classify(p[r]);
            if (b >= B)
                set_status(status, GF_INVALID);
            else
                bp[r] = b;
        }
    }
    // 2. stable rank inside the tile, per-bin tile totals
    warp_rank<Shape>(bp, warp_cnt, B);
    __syncthreads();
    warp_offsets<Shape>(warp_cnt, bin_tot, B);
    __syncthreads();

    // 3. publish the tile aggregate, then look back (inside the batch) for the exclusive prefixes
    unsigned long long* my_desc = mb.desc + (size_t)t * B;
    for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads)
        st_relaxed_u64(my_desc + b, make_desc(epoch, t == 0 ? 2u : 1u, bin_tot[b]));
    const uint32_t n_valid = block_exclusive_scan<Shape::kThreads>(bin_tot, bin_excl, B, scan_tmp);

    // 4. updater, stage in bin order
#pragma unroll
    for (int r = 0; r < Shape::kIpt; ++r) {
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

    // 5. look-back
    if (t != 0u)
        block_lookback<Shape::kThreads>(mb.desc, t, B, epoch, gbase, chunk_lo, lb_flag, lb_val, status);
    else
        for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads)
            gbase[b] = 0u;
    __syncthreads();

    // 6. inclusive prefixes, batch totals, output chunks by first-touch claim
    for (uint32_t b = threadIdx.x; b < B; b += Shape::kThreads) {
        const uint32_t excl = gbase[b], tot = bin_tot[b];
        if (t != 0u)
            st_relaxed_u64(my_desc + b, make_desc(epoch, 2u, excl + tot));
        if (t + 1u == mb.n_tiles)
            mb.totals[b] = excl + tot;
        gbase[b] = excl - bin_excl[b];
        uint32_t lo = kNoChunk, hi = kNoChunk;
        if (tot != 0u) {
            const uint32_t ka = fdc.div(excl), kb = fdc.div(excl + tot - 1u);
            k0[b] = ka;
            if (kb >= max_k) {
                set_status(status, GF_OVERFLOW);
            } else {
                lo = claim_chunk(mb.port_chunks + (size_t)b * max_k + ka, epoch, mb.counters, mb.reserved,
                                 mb.n_reserved, status);
                if (kb != ka)
                    hi = claim_chunk(mb.port_chunks + (size_t)b * max_k + kb, epoch, mb.counters, mb.reserved,
                                     mb.n_reserved, status);
            }
        }
        chunk_lo[b] = lo;
        chunk_hi[b] = hi;
    }
    if (threadIdx.x == 0)
        s_tile[2] = ld_relaxed_u32(status);
    __syncthreads();
    if (s_tile[2] != 0u) {
        retire(); // the launch failed somewhere: write nothing, the host discards every batch
        return;
    }

    // 7. coalesced write-out
    for (uint32_t q = threadIdx.x; q < n_valid; q += Shape::kThreads) {
        const uint32_t b = stage_bin[q];
        const uint32_t j = gbase[b] + q;
        const uint32_t k = fdc.div(j);
        const uint32_t chunk = k == k0[b] ? chunk_lo[b] : chunk_hi[b];
        if (chunk == kNoChunk)
            continue;
        const uint64_t slot = (uint64_t)chunk * capacity + (j - k * capacity);
        if (slot < pool_slots)
            acc.store(slot, stage[q]);
        else
            set_status(status, GF_OVERFLOW);
    }
    retire();
}

// Device form of planDenseBins + buildDenseTable + the output-descriptor loop
// (DenseBinTable.hpp:39-91, Execution.hpp:2558-2581) for a fused launch. One CTA.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) fused_finish_kernel(const uint32_t* totals,
                                                               const unsigned long long* port_chunks, uint32_t B,
                                                               uint32_t capacity, FastDiv fdc, uint32_t max_k,
                                                               const FusedCtl* ctl, uint32_t* table, gf_out_desc* descs,
                                                               uint32_t desc_cap, uint32_t* num_out, uint32_t* status)
{
    extern __shared__ uint32_t smem[];
    uint32_t* nck = smem;         // [4096]
    uint32_t* base = nck + 4096;  // [4096]
    uint32_t* tmp = base + 4096;  // [W+1]
    finish_plan<THREADS>(totals, port_chunks, B, capacity, fdc, max_k, ctl->epoch, table, descs, desc_cap, num_out,
                         status, nck, base, 4096u, tmp);
}

// Synthetic key source (uniform / Zipf / one port / round robin) at stream positions
// (first_id + i, 0, 0x100 + dist).
static __global__ void generate_keys_kernel(int dist, uint64_t seed_mixed, uint64_t first_id, uint64_t n, uint32_t bins,
                                     const double* cdf, uint32_t* keys)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = synthetic_key(dist, seed_mixed, first_id + i, bins, cdf);
}

} // namespace
} // namespace gf
