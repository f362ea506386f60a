// Hash-bin partition kernels (large port counts) and the device-side exact plan.
//
// Reference behaviour restated (paths inside graphFlow's include/graphFlow):
//   table         graph/BinTable.hpp:29-137 (open addressing, key = bin id, slot = bin * 0x9E3779B1
//                 masked, linear probing, atomicCas insert; a full table is a batch error)
//   classify      flow/Execution.hpp:1208-1307, graph/HashClassifyKernel.hpp:35-117
//   scatter       flow/Execution.hpp:1336-1502, graph/HashScatterKernel.hpp:34-183
//   plan          graph/DenseBinTable.hpp:39-91 and Execution.hpp:2558-2590 (device form here)
//
// B200 form: the table has 2 x tile entries (so it cannot fill), inserts are warp-aggregated (one
// CAS + one add per distinct bin per warp round), the tile is staged in shared memory grouped by
// entry and written out so that items of one port land on consecutive slots.
#pragma once

#include "gf_partition.cuh"

namespace gf {
namespace { // internal linkage: see gf_partition.cuh

struct alignas(16) Rec16 {
    uint64_t key;
    float weight;
    uint32_t tag;
};
static_assert(sizeof(Rec16) == 16, "16-byte record");

// SoA: three columns (u64 key, f32 weight, u32 tag).
struct Rec16SoA {
    using Payload = Rec16;
    const uint64_t* key_in;
    const float* w_in;
    const uint32_t* tag_in;
    uint64_t* key_out;
    float* w_out;
    uint32_t* tag_out;
    GF_D Payload load(uint64_t s) const { return Rec16{ld_stream(key_in + s), ld_stream(w_in + s), ld_stream(tag_in + s)}; }
    GF_D uint64_t load_key(uint64_t s) const { return ld_stream(key_in + s); }
    GF_D void store(uint64_t s, const Payload& p) const
    {
        key_out[s] = p.key;
        w_out[s] = p.weight;
        tag_out[s] = p.tag;
    }
};

// AoS: one 16-byte record per slot.
struct Rec16AoS {
    using Payload = Rec16;
    const Rec16* in;
    Rec16* out;
    GF_D Payload load(uint64_t s) const
    {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(in + s));
        Rec16 r;
        r.key = ((uint64_t)v.y << 32) | v.x;
        r.weight = __uint_as_float(v.z);
        r.tag = v.w;
        return r;
    }
    GF_D uint64_t load_key(uint64_t s) const { return __ldg(reinterpret_cast<const unsigned long long*>(in + s)); }
    GF_D void store(uint64_t s, const Payload& p) const
    {
        uint4 v;
        v.x = (uint32_t)p.key;
        v.y = (uint32_t)(p.key >> 32);
        v.z = __float_as_uint(p.weight);
        v.w = p.tag;
        *reinterpret_cast<uint4*>(out + s) = v;
    }
};

// Port of a mixed key: rank = unmix64(key) ^ salt; a rank >= bins is invalid.
struct UnmixClassify {
    uint64_t salt;
    uint32_t bins;
    GF_HD uint32_t operator()(uint64_t key) const
    {
        const uint64_t r = unmix64(key) ^ salt;
        return r < bins ? (uint32_t)r : bins;
    }
};

constexpr uint32_t kHashEmpty = 0xFFFFFFFFu; // graph/BinTable.hpp:29-32

GF_HD uint32_t hash_slot(uint32_t bin, uint32_t mask) { return (bin * 0x9E3779B1u) & mask; } // BinTable.hpp:90-93

// Warp-aggregated insert of this lane's bin (kNoBin lanes take part but insert nothing).
// Returns the entry index (or kNoChunk when the table is full) and the item's rank among the
// items of its bin inserted so far (arrival order).
GF_D void hash_insert_warp(uint32_t bin, uint32_t* hkey, uint32_t* hcnt, uint32_t mask, uint32_t& entry,
                           uint32_t& rank)
{
    const int lane = threadIdx.x & 31;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, bin);
    const int leader = 31 - __clz(peers);
    uint32_t e = kNoChunk, base = 0;
    if (lane == leader && bin != kNoBin) {
        uint32_t slot = hash_slot(bin, mask);
        for (uint32_t probe = 0; probe <= mask; ++probe) {
            const uint32_t old = atomicCAS(&hkey[slot], kHashEmpty, bin);
            if (old == kHashEmpty || old == bin) {
                e = slot;
                base = atomicAdd(&hcnt[slot], (uint32_t)__popc(peers));
                break;
            }
            slot = (slot + 1u) & mask;
        }
    }
    e = __shfl_sync(0xFFFFFFFFu, e, leader);
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    entry = e;
    rank = base + __popc(peers & lanemask_lt());
}

template <int E, int THREADS>
GF_D void hash_reset(uint32_t* hkey, uint32_t* hcnt)
{
    for (int i = threadIdx.x; i < E; i += THREADS) {
        hkey[i] = kHashEmpty;
        hcnt[i] = 0u;
    }
}

// ---------------------------------------------------------------------------------------------
// Hash classify: per tile, classify each key, store its bin (optional), aggregate per bin in the
// shared table, then one device atomic per occupied entry into counts[bin]. counts[bins] is the
// status slot. `bin_ids == nullptr` skips the store (device-planned form recomputes the bin).
// ---------------------------------------------------------------------------------------------
template <typename Shape, typename Access>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) hash_classify_kernel(Access acc, UnmixClassify cls,
                                                                        uint32_t capacity, uint64_t pool_slots,
                                                                        const gf_tile* tiles, uint32_t n_tiles,
                                                                        uint32_t B, uint32_t* bin_ids,
                                                                        uint32_t* counts, uint32_t* status)
{
    constexpr int E = 2 * Shape::kTile;
    __shared__ uint32_t hkey[E], hcnt[E];
    __shared__ uint32_t full;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const gf_tile tile = tiles[t];
        const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
        const bool tile_ok = tile.count <= (uint32_t)Shape::kTile && base + tile.count <= pool_slots &&
                             tile.tile_offset + tile.count <= capacity;
        hash_reset<E, Shape::kThreads>(hkey, hcnt);
        if (threadIdx.x == 0)
            full = 0u;
        __syncthreads();
        uint64_t keys[Shape::kIpt];
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            if (tile_ok && i < tile.count)
                keys[r] = acc.load_key(base + i);
        }
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            uint32_t bin = kNoBin;
            if (tile_ok && i < tile.count) {
                bin = cls(keys[r]);
                if (bin >= B) {
                    counts[B] = 1u;
                    set_status(status, GF_INVALID);
                    bin = kNoBin;
                } else if (bin_ids != nullptr) {
                    bin_ids[base + i] = bin;
                }
            }
            uint32_t e, rank;
            hash_insert_warp(bin, hkey, hcnt, E - 1, e, rank);
            if (bin != kNoBin && e == kNoChunk)
                full = 1u;
        }
        if (!tile_ok && threadIdx.x == 0)
            set_status(status, GF_INVALID);
        __syncthreads();
        if (full != 0u) {
            if (threadIdx.x == 0) {
                counts[B] = 1u;
                set_status(status, GF_ERR_TABLE_FULL);
            }
        } else {
            for (int e = threadIdx.x; e < E; e += Shape::kThreads)
                if (hkey[e] != kHashEmpty)
                    atomicAdd(&counts[hkey[e]], hcnt[e]);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Hash scatter: per tile, rebuild the table from the stored bins (or recompute them from the
// keys), reserve one range per occupied entry with atomicAdd(next[bin], count), stage the tile
// grouped by entry, apply the updater, write out through the dense table layout
// out = table[B + table[bin] + j / C] * C + j % C.
// ---------------------------------------------------------------------------------------------
template <typename Shape, typename Access, typename Update>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) hash_scatter_kernel(Access acc, UnmixClassify cls, Update update,
                                                                       uint64_t seed_mixed, uint32_t capacity,
                                                                       FastDiv fdc, uint64_t pool_slots,
                                                                       const gf_tile* tiles, uint32_t n_tiles,
                                                                       uint32_t B, const uint32_t* bin_ids,
                                                                       const uint32_t* table, uint32_t* next,
                                                                       uint32_t* counts, uint32_t* status)
{
    using P = typename Access::Payload;
    constexpr int E = 2 * Shape::kTile;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* stage = reinterpret_cast<P*>(smem_raw);                         // [TILE]
    uint32_t* stage_e = reinterpret_cast<uint32_t*>(stage + Shape::kTile); // [TILE]
    uint32_t* hkey = stage_e + Shape::kTile;                           // [E]
    uint32_t* hcnt = hkey + E;                                         // [E]
    uint32_t* hexcl = hcnt + E;                                        // [E]
    uint32_t* hgb = hexcl + E;                                         // [E]
    uint32_t* scan_tmp = hgb + E;                                      // [W+1]
    uint32_t* s_full = scan_tmp + Shape::kWarps + 1;                   // [1]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const gf_tile tile = tiles[t];
        const uint64_t base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
        const bool tile_ok = tile.count <= (uint32_t)Shape::kTile && base + tile.count <= pool_slots &&
                             tile.tile_offset + tile.count <= capacity;
        hash_reset<E, Shape::kThreads>(hkey, hcnt);
        if (threadIdx.x == 0)
            *s_full = 0u;
        __syncthreads();
        P p[Shape::kIpt];
        uint32_t ent[Shape::kIpt], rank[Shape::kIpt];
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            if (tile_ok && i < tile.count)
                p[r] = acc.load(base + i);
        }
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            uint32_t bin = kNoBin;
            if (tile_ok && i < tile.count) {
                bin = bin_ids != nullptr ? __ldg(bin_ids + base + i) : cls(p[r].key);
                if (bin >= B) {
                    counts[B] = 1u;
                    set_status(status, GF_INVALID);
                    bin = kNoBin;
                }
            }
            hash_insert_warp(bin, hkey, hcnt, E - 1, ent[r], rank[r]);
            if (bin == kNoBin)
                ent[r] = kNoChunk;
            else if (ent[r] == kNoChunk)
                *s_full = 1u;
        }
        if (!tile_ok && threadIdx.x == 0)
            set_status(status, GF_INVALID);
        __syncthreads();
        if (*s_full != 0u) {
            // HashScatterKernel.hpp:126-131: a full table is a hard batch error, nothing is written
            if (threadIdx.x == 0) {
                counts[B] = 1u;
                set_status(status, GF_ERR_TABLE_FULL);
            }
            return;
        }
        const uint32_t n_valid = block_exclusive_scan<Shape::kThreads>(hcnt, hexcl, E, scan_tmp);
        for (int e = threadIdx.x; e < E; e += Shape::kThreads)
            if (hcnt[e] != 0u)
                hgb[e] = atomicAdd(&next[hkey[e]], hcnt[e]) - hexcl[e];
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            if (ent[r] == kNoChunk)
                continue;
            const uint32_t q = hexcl[ent[r]] + rank[r];
            const uint32_t res = update(hkey[ent[r]], p[r], seed_mixed);
            if (res != kUpdateSuccess) {
                counts[B] = 1u;
                set_status(status, res == kUpdateOverflow ? GF_OVERFLOW : GF_INVALID);
            }
            stage[q] = p[r];
            stage_e[q] = ent[r];
        }
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < n_valid; q += Shape::kThreads) {
            const uint32_t e = stage_e[q];
            const uint32_t b = hkey[e];
            const uint32_t j = hgb[e] + q;
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

// ---------------------------------------------------------------------------------------------
// Device plan from the per-bin totals and a reservation: binBase = exclusive scan of
// ceil(total_b / C) (DenseBinTable.hpp:39-77), chunk (b, k) = reserved[binBase[b] + k],
// table = [binBase[B], chunkIndex[R]] (DenseBinTable.hpp:80-91), descriptors in bin order with
// their fills (Execution.hpp:2558-2581), next[] zeroed for the scatter. One CTA.
// counts[B] (the classify status slot) must be zero; the plan also checks R <= n_reserved.
// ---------------------------------------------------------------------------------------------
template <int THREADS>
__global__ void __launch_bounds__(THREADS) plan_device_kernel(const uint32_t* counts, uint32_t B, uint32_t capacity,
                                                              FastDiv fdc, const uint32_t* reserved,
                                                              uint32_t n_reserved, uint32_t* table,
                                                              gf_out_desc* descs, uint32_t desc_cap,
                                                              uint32_t* num_out, uint32_t* next, uint32_t* status)
{
    __shared__ uint32_t tmp[THREADS / 32 + 1];
    __shared__ uint32_t s_part[THREADS];
    if (counts[B] != 0u) {
        if (threadIdx.x == 0) {
            set_status(status, GF_INVALID);
            *num_out = 0u;
        }
        return;
    }
    // contiguous segment per thread
    const uint32_t per = (B + THREADS - 1) / THREADS;
    const uint32_t lo = min(B, threadIdx.x * per), hi = min(B, lo + per);
    uint32_t sum = 0;
    for (uint32_t b = lo; b < hi; ++b) {
        const uint32_t c = counts[b];
        sum += fdc.div(c) + (fdc.mod(c) != 0u ? 1u : 0u);
    }
    s_part[threadIdx.x] = sum;
    __syncthreads();
    const uint32_t total = block_exclusive_scan<THREADS>(s_part, s_part, THREADS, tmp);
    if (total > n_reserved || total > desc_cap) {
        if (threadIdx.x == 0) {
            set_status(status, GF_OVERFLOW);
            *num_out = 0u;
        }
        return;
    }
    uint32_t run = s_part[threadIdx.x];
    for (uint32_t b = lo; b < hi; ++b) {
        const uint32_t c = counts[b];
        const uint32_t nk = fdc.div(c) + (fdc.mod(c) != 0u ? 1u : 0u);
        table[b] = run;
        next[b] = 0u;
        for (uint32_t k = 0; k < nk; ++k) {
            const uint32_t chunk = __ldg(reserved + run + k);
            table[B + run + k] = chunk;
            descs[run + k].chunk_index = chunk;
            descs[run + k].fill = min(capacity, c - k * capacity);
            descs[run + k].bin = b;
        }
        run += nk;
    }
    if (threadIdx.x == 0)
        *num_out = total;
}

// Synthetic 16-byte records: rank r ~ Zipf(cdf over k), key = mix64(r ^ salt), weight = U(0,1]
// f32, tag = id; stream position (first_id + i, 0, 0x110), draws 0 and 1.
template <typename Access>
__global__ void generate_records16_kernel(Access acc, uint64_t seed_mixed, uint64_t first_id, uint64_t n,
                                          const double* cdf, uint32_t k, uint64_t salt)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t id = first_id + i;
        const Philox4 d = first_draws(stream_key(seed_mixed, id, 0u, 0x110u));
        const double u = uniform_f64(d.v[0]);
        uint32_t lo = 0, hi = k - 1u;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2u;
            if (u < cdf[mid])
                hi = mid;
            else
                lo = mid + 1u;
        }
        Rec16 r;
        r.key = mix64((uint64_t)lo ^ salt);
        r.weight = 1.0f - uniform_f32(d.v[1]);
        r.tag = (uint32_t)id;
        acc.store(i, r);
    }
}

} // namespace
} // namespace gf
