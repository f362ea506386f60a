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

#include <type_traits>

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
// The per-tile kernels take the C ABI's key classifier (UnmixClassify: only the 8-byte key is
// loaded) or any classifier of a whole payload (the front end's partition stages).
template <typename Cls>
inline constexpr bool kKeyClassifier = std::is_same_v<Cls, UnmixClassify>;

template <typename Cls, typename P>
GF_D uint32_t hash_bin_of(const Cls& cls, const P& p)
{
    if constexpr (kKeyClassifier<Cls>)
        return cls(p.key);
    else
        return cls(p);
}

template <typename Shape, typename Access, typename Cls = UnmixClassify>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) hash_classify_kernel(Access acc, Cls cls,
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
        using In = std::conditional_t<kKeyClassifier<Cls>, uint64_t, typename Access::Payload>;
        In keys[Shape::kIpt];
#pragma unroll
        for (int r = 0; r < Shape::kIpt; ++r) {
            const uint32_t i = Shape::item(w, r, lane);
            if (tile_ok && i < tile.count) {
                if constexpr (kKeyClassifier<Cls>)
                    keys[r] = acc.load_key(base + i);
                else
                    keys[r] = acc.load(base + i);
            }
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
template <typename Shape, typename Access, typename Update, typename Cls = UnmixClassify>
__global__ void __launch_bounds__(Shape::kThreads, Shape::kMinBlocks) hash_scatter_kernel(Access acc, Cls cls, Update update,
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
                bin = bin_ids != nullptr ? __ldg(bin_ids + base + i) : hash_bin_of(cls, p[r]);
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
// Persistent form of hash classify and scatter. The ports of this path are dense ranks
// (unmix64(key) ^ salt < bins), so no per-tile open-addressing table is needed: every CTA owns a
// contiguous range of tiles and keeps, for the ports below kHashSmemBins, one shared-memory
// counter per port for its whole range (one device atomic per CTA and port instead of one per
// tile and port); a record of a port at or above kHashSmemBins goes to a device atomic directly.
// The scatter (hash_scatter_grouped_kernel below) writes through the dense table layout
// out = table[B + table[port] + j / C] * C + j % C.
// ---------------------------------------------------------------------------------------------
constexpr uint32_t kHashSmemBins = 8192u;
constexpr uint32_t kHashGroupBins = 2048u; // up to this many ports the scatter groups each tile by port
constexpr int kHashPThreads = 256;
constexpr int kHashPUnroll = 4; // records per thread in flight

GF_D bool hash_tile_range(const gf_tile* tiles, uint32_t t, uint32_t capacity, uint64_t pool_slots, uint64_t& base,
                          uint32_t& count, uint32_t* status)
{
    const gf_tile tile = tiles[t];
    base = (uint64_t)tile.chunk_index * capacity + tile.tile_offset;
    const bool ok = base + tile.count <= pool_slots && tile.tile_offset + tile.count <= capacity;
    if (!ok && threadIdx.x == 0)
        set_status(status, GF_INVALID);
    count = ok ? tile.count : 0u;
    return ok;
}

// Counts of ports [0, ks) of this CTA's range into hist (zeroed here); ports >= ks go to
// counts[] directly. With bin_ids, every record's port is stored.
template <typename Access>
GF_D void hash_count_range(const Access& acc, const UnmixClassify& cls, uint32_t capacity, uint64_t pool_slots,
                           const gf_tile* tiles, uint32_t t_lo, uint32_t t_hi, uint32_t B, uint32_t ks,
                           uint32_t* bin_ids, uint32_t* hist, uint32_t* counts, uint32_t* status)
{
    for (uint32_t i = threadIdx.x; i < ks; i += blockDim.x)
        hist[i] = 0u;
    __syncthreads();
    bool bad = false;
    for (uint32_t t = t_lo; t < t_hi; ++t) {
        uint64_t base;
        uint32_t count;
        hash_tile_range(tiles, t, capacity, pool_slots, base, count, status);
        for (uint32_t i0 = 0; i0 < count; i0 += kHashPThreads * kHashPUnroll) {
            uint64_t key[kHashPUnroll];
#pragma unroll
            for (int u = 0; u < kHashPUnroll; ++u) {
                const uint32_t i = i0 + (uint32_t)u * kHashPThreads + threadIdx.x;
                key[u] = i < count ? acc.load_key(base + i) : 0ull;
            }
#pragma unroll
            for (int u = 0; u < kHashPUnroll; ++u) {
                const uint32_t i = i0 + (uint32_t)u * kHashPThreads + threadIdx.x;
                if (i >= count)
                    continue;
                const uint32_t b = cls(key[u]);
                if (b >= B) {
                    bad = true;
                    continue;
                }
                if (bin_ids != nullptr)
                    bin_ids[base + i] = b;
                if (b < ks)
                    atomicAdd(&hist[b], 1u);
                else
                    atomicAdd(&counts[b], 1u);
            }
        }
    }
    if (bad) {
        counts[B] = 1u;
        set_status(status, GF_INVALID);
    }
    __syncthreads();
}

template <typename Access>
__global__ void __launch_bounds__(kHashPThreads) hash_count_persist_kernel(Access acc, UnmixClassify cls,
                                                                           uint32_t capacity, uint64_t pool_slots,
                                                                           const gf_tile* tiles, uint32_t n_tiles,
                                                                           uint32_t B, uint32_t* bin_ids,
                                                                           uint32_t* counts, uint32_t* status)
{
    extern __shared__ uint32_t hist[]; // [ks]
    const uint32_t ks = B < kHashSmemBins ? B : kHashSmemBins;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    const uint32_t t_lo = (uint32_t)((uint64_t)n_tiles * c / G), t_hi = (uint32_t)((uint64_t)n_tiles * (c + 1u) / G);
    hash_count_range(acc, cls, capacity, pool_slots, tiles, t_lo, t_hi, B, ks, bin_ids, hist, counts, status);
    for (uint32_t b = threadIdx.x; b < ks; b += blockDim.x)
        if (hist[b] != 0u)
            atomicAdd(&counts[b], hist[b]);
}

// Grouped scatter: persistent CTAs over contiguous tile ranges, processed in units of up to
// `unit` records (unit / 256 rows; a row is up to 256 consecutive records of one tile, so a unit
// spans several small tiles). In every unit the records of ports below GB = min(B, kHashGroupBins)
// are grouped by port in shared memory: a direct-indexed count per port gives each record its
// rank, an exclusive scan over the GB ports its stage position, each port present in the unit
// reserves its range with one device atomic on next[port] (arrival order between units, as
// graph/HashScatterKernel.hpp:132-150 reserves per table entry), and a port's records of the unit
// go to consecutive slots from consecutive threads. A record of a port >= GB (the tail of a
// popularity-ranked key space; compiled only when B > kHashGroupBins, kTail) is staged at the end
// of the unit's stage and reserves its own slot with one device atomic.
//
// A record is staged at its input position as soon as it is classified (its registers are free for
// the scan); the stage step only writes, per port-order position, the record's input position.
// Thread t owns ports t, t + 256, ... (PPT of them; the popular low ports spread over all warps):
// it scans their counts and issues their reservations before the stage step, which hides the
// atomics' latency behind a barrier and the staging. Warp 0 prefetches the next unit's tile
// descriptors with cp.async while the unit's records are counted, and builds its row table from
// them. The tail's reservations are issued at the same point and consumed after the grouped
// write-out.
constexpr uint32_t kHashRowsEnd = 0xFFFFFFFFu;
constexpr uint32_t kHashTailEarly = 2u; // tail records per thread reserved ahead of the write-out

GF_D void cp_async4(void* smem_dst, const void* gmem_src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
                 "l"(gmem_src)
                 : "memory");
}
GF_D void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
GF_D void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Warp 0: copy the descriptors of tiles cur_t .. cur_t + nr_max - 1 (those below t_hi) into tstage.
GF_D void hash_prefetch_tiles(const gf_tile* tiles, uint32_t t_hi, uint32_t nr_max, uint32_t cur_t, uint32_t* tstage)
{
    const uint32_t lane = threadIdx.x & 31u;
    if (cur_t < t_hi && lane < nr_max && lane < t_hi - cur_t) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(tiles + cur_t + lane);
        cp_async4(tstage + 3u * lane, src);
        cp_async4(tstage + 3u * lane + 1u, src + 1);
        cp_async4(tstage + 3u * lane + 2u, src + 2);
    }
    cp_async_commit();
}

// Warp 0 (every lane keeps the same cursor): row table of the unit that starts at tile cur_t,
// record cur_off, from the descriptors prefetched into tstage. Rows are taken in tile order up to
// nr_max; the cursor moves past them.
GF_D void hash_build_rows(uint32_t t_hi, uint32_t capacity, uint64_t pool_slots, uint32_t nr_max, uint32_t& cur_t,
                          uint32_t& cur_off, const uint32_t* tstage, uint64_t* rbase, uint32_t* rcnt, uint32_t* nrows,
                          uint32_t* status)
{
    constexpr uint32_t T = kHashPThreads;
    const uint32_t lane = threadIdx.x & 31u;
    cp_async_wait_all();
    __syncwarp();
    if (cur_t >= t_hi) {
        if (lane == 0u)
            *nrows = kHashRowsEnd;
        return;
    }
    const uint32_t loaded = t_hi - cur_t < nr_max ? t_hi - cur_t : nr_max;
    uint64_t base = 0;
    uint32_t rows = 0, rem = 0, off = 0;
    if (lane < loaded) {
        const uint32_t chunk = tstage[3u * lane], toff = tstage[3u * lane + 1u], tcount = tstage[3u * lane + 2u];
        base = (uint64_t)chunk * capacity + toff;
        const bool ok = base + tcount <= pool_slots && (uint64_t)toff + tcount <= capacity;
        if (!ok)
            set_status(status, GF_INVALID);
        const uint32_t count = ok ? tcount : 0u;
        off = lane == 0u ? cur_off : 0u;
        rem = count > off ? count - off : 0u;
        rows = (rem + T - 1u) / T;
    }
    uint32_t incl = rows;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((int)lane >= o)
            incl += y;
    }
    const uint32_t excl = incl - rows;
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    for (uint32_t j = excl; j < incl && j < nr_max; ++j) {
        const uint32_t k = j - excl;
        rbase[j] = base + off + (uint64_t)k * T;
        rcnt[j] = rem - k * T < T ? rem - k * T : T;
    }
    if (total <= nr_max) {
        cur_t += loaded;
        cur_off = 0u;
    } else {
        const uint32_t L = (uint32_t)__ffs(__ballot_sync(0xFFFFFFFFu, incl >= nr_max)) - 1u;
        const uint32_t ex = __shfl_sync(0xFFFFFFFFu, excl, L), in = __shfl_sync(0xFFFFFFFFu, incl, L);
        const uint32_t of = __shfl_sync(0xFFFFFFFFu, off, L);
        if (in == nr_max) {
            cur_t += L + 1u;
            cur_off = 0u;
        } else {
            cur_t += L;
            cur_off = of + (nr_max - ex) * T;
        }
    }
    if (lane == 0u)
        *nrows = total < nr_max ? total : nr_max;
    __syncwarp(); // tstage is refilled by the next prefetch
}

// With more than 1024 grouped ports the port arrays take 24 KB: three CTAs per SM, whose register
// bound then leaves room for the eight owned ports.
template <typename Access, typename Update, bool kTail, uint32_t PPT>
__global__ void __launch_bounds__(kHashPThreads, PPT == 8u ? 3 : 4) hash_scatter_grouped_kernel(
    Access acc, UnmixClassify cls, Update update, uint64_t seed_mixed, uint32_t capacity, FastDiv fdc,
    uint64_t pool_slots, const gf_tile* tiles, uint32_t n_tiles, uint32_t B, uint32_t unit, const uint32_t* bin_ids,
    const uint32_t* table, uint32_t* next, uint32_t* counts, uint32_t* status)
{
    using P = typename Access::Payload;
    using SPort = std::conditional_t<kTail, uint32_t, uint16_t>;
    constexpr uint32_t T = kHashPThreads, W = T / 32u, RPT = 2048u / T; // rows per unit: unit / T <= RPT
    static_assert((PPT == 4u || PPT == 8u) && PPT * T >= kHashGroupBins / 2u && (!kTail || PPT * T >= kHashGroupBins),
                  "owned ports: PPT per thread cover the grouped ports");
    extern __shared__ __align__(128) uint32_t sm[];
    const uint32_t GB = B < kHashGroupBins ? B : kHashGroupBins;
    P* stage = reinterpret_cast<P*>(sm);                              // [unit]
    uint64_t* rbase = reinterpret_cast<uint64_t*>(stage + unit);      // [2][RPT]
    uint32_t* tc = reinterpret_cast<uint32_t*>(rbase + 2u * RPT);     // [GB] count | stage start << 16
    uint32_t* D = tc + GB;                                            // [GB] reserved position - stage start
    uint32_t* PB = D + GB;                                            // [GB] table[port]
    uint32_t* rcnt = PB + GB;                                         // [2][RPT]
    uint32_t* nrows = rcnt + 2u * RPT;                                // [2]
    uint32_t* ntail = nrows + 2u;                                     // [2]
    uint32_t* scan_tmp = ntail + 2u;                                  // [PPT][W]
    uint32_t* tstage = scan_tmp + PPT * W;                            // [3 * RPT] prefetched tile descriptors
    SPort* sport = reinterpret_cast<SPort*>(tstage + 3u * RPT);       // [unit] port per output position
    uint16_t* src = reinterpret_cast<uint16_t*>(sport + unit);        // [unit] input position per output position
    const uint32_t tid = threadIdx.x, w = tid >> 5, lane = tid & 31u;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    const uint32_t t_lo = (uint32_t)((uint64_t)n_tiles * c / G), t_hi = (uint32_t)((uint64_t)n_tiles * (c + 1u) / G);
    const uint32_t nr_max = unit / T;
    for (uint32_t i = tid; i < GB; i += T) {
        tc[i] = 0u;
        PB[i] = __ldg(table + i);
    }
    uint32_t cur_t = t_lo, cur_off = 0u;
    if (w == 0u) {
        hash_prefetch_tiles(tiles, t_hi, nr_max, cur_t, tstage);
        hash_build_rows(t_hi, capacity, pool_slots, nr_max, cur_t, cur_off, tstage, rbase, rcnt, nrows, status);
    }
    if (tid == 0u)
        ntail[0] = ntail[1] = 0u;
    __syncthreads();
    bool bad = false, overflow = false;
    uint32_t upd = kUpdateSuccess;
    for (uint32_t it = 0;; ++it) {
        const uint32_t buf = it & 1u;
        const uint32_t nr = nrows[buf];
        if (nr == kHashRowsEnd)
            break;
        P rec[RPT];
        uint32_t bp[RPT];   // port | rank << 16 of a grouped record, else kNoBin16
        uint32_t valid = 0; // bit r: this thread has a record in row r
#pragma unroll
        for (uint32_t r = 0; r < RPT; ++r) {
            if (r < nr && tid < rcnt[buf * RPT + r]) {
                valid |= 1u << r;
                rec[r] = acc.load(rbase[buf * RPT + r] + tid);
            }
        }
        // the next unit's tile descriptors arrive while this unit is counted and staged
        if (w == 0u)
            hash_prefetch_tiles(tiles, t_hi, nr_max, cur_t, tstage);
        if (tid == 0u)
            ntail[buf ^ 1u] = 0u; // its last reader (the previous unit's write-out) is past a barrier
#pragma unroll
        for (uint32_t r = 0; r < RPT; ++r) {
            bp[r] = kNoBin16;
            if (valid & (1u << r)) {
                const uint32_t b = bin_ids != nullptr ? __ldg(bin_ids + rbase[buf * RPT + r] + tid) : cls(rec[r].key);
                if (b < GB) {
                    bp[r] = b | ((atomicAdd(&tc[b], 1u) & 0xFFFFu) << 16);
                } else if (kTail && b < B) {
                    const uint32_t q = unit - 1u - atomicAdd(&ntail[buf], 1u);
                    src[q] = (uint16_t)(r * T + tid);
                    sport[q] = (SPort)b;
                } else {
                    bad = true;
                    continue;
                }
                const uint32_t res = update(b, rec[r], seed_mixed);
                if (res != kUpdateSuccess)
                    upd = res;
                stage[r * T + tid] = rec[r];
            }
        }
        __syncthreads();
        // exclusive scan over the grouped ports in port order: one warp scan per owned column
        // (and each owned port's reservation, issued as soon as its count is final)
        uint32_t cw[PPT], incl[PPT], j0[PPT];
#pragma unroll
        for (uint32_t i = 0; i < PPT; ++i) {
            const uint32_t p = tid + i * T;
            cw[i] = p < GB ? tc[p] & 0xFFFFu : 0u;
            incl[i] = cw[i];
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
            for (uint32_t i = 0; i < PPT; ++i) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl[i], o);
                if ((int)lane >= o)
                    incl[i] += y;
            }
        }
        if (lane == 31u) {
#pragma unroll
            for (uint32_t i = 0; i < PPT; ++i)
                scan_tmp[i * W + w] = incl[i];
        }
        // the tail's reservations: all tail records of the unit are staged by now
        uint32_t tj[kHashTailEarly], tpb[kHashTailEarly];
        uint32_t nt = 0;
        if constexpr (kTail) {
            nt = ntail[buf];
#pragma unroll
            for (uint32_t u = 0; u < kHashTailEarly; ++u) {
                const uint32_t i = u * T + tid;
                const uint32_t b = i < nt ? (uint32_t)sport[unit - 1u - i] : 0u;
                tj[u] = i < nt ? atomicAdd(&next[b], 1u) : 0u;
                tpb[u] = i < nt ? __ldg(table + b) : 0u;
            }
        }
        __syncthreads();
        uint32_t n_grouped = 0;
#pragma unroll
        for (uint32_t i = 0; i < PPT; ++i) {
            uint32_t pre = n_grouped; // ports of the columns before, and of the warps before in this column
#pragma unroll
            for (uint32_t v = 0; v < W; ++v) {
                const uint32_t x = scan_tmp[i * W + v];
                pre += v < w ? x : 0u;
                n_grouped += x;
            }
            const uint32_t start = pre + incl[i] - cw[i];
            const uint32_t p = tid + i * T;
            j0[i] = cw[i] != 0u ? atomicAdd(&next[p], cw[i]) : 0u;
            if (p < GB)
                tc[p] = start << 16; // the stage start replaces the count
            cw[i] = cw[i] != 0u ? start : 0xFFFFFFFFu;
        }
        __syncthreads();
        // the grouped records in port order: output position -> input position and port
#pragma unroll
        for (uint32_t r = 0; r < RPT; ++r) {
            const uint32_t b = bp[r] & 0xFFFFu;
            if (b != kNoBin16) {
                const uint32_t q = (tc[b] >> 16) + (bp[r] >> 16);
                src[q] = (uint16_t)(r * T + tid);
                sport[q] = (SPort)b;
            }
        }
#pragma unroll
        for (uint32_t i = 0; i < PPT; ++i)
            if (cw[i] != 0xFFFFFFFFu)
                D[tid + i * T] = j0[i] - cw[i];
        // the next unit's rows (the row table this unit read is past two barriers)
        if (w == 0u)
            hash_build_rows(t_hi, capacity, pool_slots, nr_max, cur_t, cur_off, tstage, rbase + (buf ^ 1u) * RPT,
                            rcnt + (buf ^ 1u) * RPT, nrows + (buf ^ 1u), status);
        __syncthreads();
        // write-out: grouped positions [0, n_grouped), then the tail [unit - n_tail, unit)
        constexpr uint32_t kU = 4u;
        for (uint32_t q0 = 0; q0 < n_grouped; q0 += kU * T) {
#pragma unroll
            for (uint32_t u = 0; u < kU; ++u) {
                const uint32_t q = q0 + u * T + tid;
                if (q < n_grouped) {
                    const uint32_t b = sport[q];
                    const uint32_t j = D[b] + q;
                    const uint32_t k = fdc.div(j);
                    const uint32_t chunk = __ldg(table + B + PB[b] + k);
                    const uint64_t slot = (uint64_t)chunk * capacity + (j - k * capacity);
                    if (slot < pool_slots)
                        acc.store(slot, stage[src[q]]);
                    else
                        overflow = true;
                }
            }
        }
        if constexpr (kTail) {
            auto put_tail = [&](uint32_t i, uint32_t j, uint32_t pbase) {
                const uint32_t k = fdc.div(j);
                const uint32_t chunk = __ldg(table + B + pbase + k);
                const uint64_t slot = (uint64_t)chunk * capacity + (j - k * capacity);
                if (slot < pool_slots)
                    acc.store(slot, stage[src[unit - 1u - i]]);
                else
                    overflow = true;
            };
#pragma unroll
            for (uint32_t u = 0; u < kHashTailEarly; ++u)
                if (u * T + tid < nt)
                    put_tail(u * T + tid, tj[u], tpb[u]);
            for (uint32_t i = kHashTailEarly * T + tid; i < nt; i += T) {
                const uint32_t b = sport[unit - 1u - i];
                put_tail(i, atomicAdd(&next[b], 1u), __ldg(table + b));
            }
        }
        __syncthreads();
    }
    if (bad || upd != kUpdateSuccess) {
        counts[B] = 1u;
        set_status(status, bad || upd == kUpdateInvalid ? GF_INVALID : GF_OVERFLOW);
    }
    if (overflow)
        set_status(status, GF_OVERFLOW);
}

// Shared memory of hash_scatter_grouped_kernel for `bins` ports and units of `unit` records.
inline size_t hash_grouped_smem(uint32_t bins, uint32_t unit)
{
    constexpr size_t rpt = 2048u / kHashPThreads, w = kHashPThreads / 32u;
    const size_t gb = bins < kHashGroupBins ? bins : kHashGroupBins;
    const size_t ppt = bins > kHashGroupBins / 2u ? 8u : 4u;
    const size_t port_bytes = (bins > kHashGroupBins ? sizeof(uint32_t) : sizeof(uint16_t)) + sizeof(uint16_t);
    return sizeof(Rec16) * unit + sizeof(uint64_t) * 2u * rpt + sizeof(uint32_t) * 3u * gb +
           sizeof(uint32_t) * (2u * rpt + 4u + ppt * w + 3u * rpt) + port_bytes * unit;
}

// ---------------------------------------------------------------------------------------------
// Device plan from the per-bin totals and a reservation: binBase = exclusive scan of
// ceil(total_b / C) (DenseBinTable.hpp:39-77), chunk (b, k) = reserved[binBase[b] + k],
// table = [binBase[B], chunkIndex[R]] (DenseBinTable.hpp:80-91), descriptors in bin order with
// their fills (Execution.hpp:2558-2581), next[] zeroed for the scatter.
// counts[B] (the classify status slot) must be zero; the plan also checks R <= n_reserved.
// Four grid-wide steps, so that the cost does not grow with B on one CTA:
//   A  block sums of ceil(total_b / C) over blocks of kPlanBlock bins, into next[block];
//   B  one CTA: exclusive scan of the block sums in place, R, the checks, num_out;
//   C  per block: binBase of every bin into table[b], next[b] = 0 for b >= #blocks;
//   D  one thread per output chunk r < R: its bin by binary search over table[0, B), the chunk id
//      and the descriptor; next[0, #blocks) = 0.
// A failed batch (status set) leaves table, descriptors and next untouched after step B.
// ---------------------------------------------------------------------------------------------
constexpr uint32_t kPlanThreads = 256u, kPlanPerThread = 8u, kPlanBlock = kPlanThreads * kPlanPerThread;

GF_D uint32_t chunks_of(uint32_t c, FastDiv fdc) { return fdc.div(c) + (fdc.mod(c) != 0u ? 1u : 0u); }

// Sum of v over the CTA, valid in every thread.
GF_D uint32_t plan_block_sum(uint32_t v, uint32_t* tmp)
{
    v = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31u) == 0u)
        tmp[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t s = 0;
    for (uint32_t i = 0; i < blockDim.x / 32u; ++i)
        s += tmp[i];
    __syncthreads();
    return s;
}

__global__ void __launch_bounds__(kPlanThreads) plan_blocksum_kernel(const uint32_t* counts, uint32_t B, FastDiv fdc,
                                                                      uint32_t* next)
{
    __shared__ uint32_t tmp[kPlanThreads / 32];
    const uint32_t b0 = blockIdx.x * kPlanBlock + threadIdx.x * kPlanPerThread;
    uint32_t s = 0;
#pragma unroll
    for (uint32_t i = 0; i < kPlanPerThread; ++i)
        if (b0 + i < B)
            s += chunks_of(counts[b0 + i], fdc);
    s = plan_block_sum(s, tmp);
    if (threadIdx.x == 0)
        next[blockIdx.x] = s;
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) plan_scan_kernel(const uint32_t* counts, uint32_t B, uint32_t n_blocks,
                                                            uint32_t n_reserved, uint32_t desc_cap, uint32_t* next,
                                                            uint32_t* num_out, uint32_t* status)
{
    __shared__ uint32_t tmp[THREADS / 32 + 1];
    const uint32_t total = block_exclusive_scan<THREADS>(next, next, n_blocks, tmp);
    if (threadIdx.x == 0) {
        if (counts[B] != 0u) {
            set_status(status, GF_INVALID);
            *num_out = 0u;
        } else if (total > n_reserved || total > desc_cap) {
            set_status(status, GF_OVERFLOW);
            *num_out = 0u;
        } else {
            *num_out = total;
        }
    }
}

__global__ void __launch_bounds__(kPlanThreads) plan_bins_kernel(const uint32_t* counts, uint32_t B, FastDiv fdc,
                                                                  uint32_t n_blocks, uint32_t* table, uint32_t* next,
                                                                  const uint32_t* status)
{
    __shared__ uint32_t tmp[kPlanThreads / 32 + 1];
    if (ld_relaxed_u32(status) != 0u)
        return;
    const uint32_t b0 = blockIdx.x * kPlanBlock + threadIdx.x * kPlanPerThread;
    uint32_t nk[kPlanPerThread], s = 0;
#pragma unroll
    for (uint32_t i = 0; i < kPlanPerThread; ++i) {
        nk[i] = b0 + i < B ? chunks_of(counts[b0 + i], fdc) : 0u;
        s += nk[i];
    }
    // exclusive prefix of s over the CTA
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((int)lane >= o)
            incl += y;
    }
    if (lane == 31u)
        tmp[w] = incl;
    __syncthreads();
    uint32_t run = next[blockIdx.x] + incl - s; // every CTA reads its base before any CTA could reuse the word
#pragma unroll
    for (uint32_t i = 0; i < kPlanThreads / 32u; ++i)
        run += i < w ? tmp[i] : 0u;
#pragma unroll
    for (uint32_t i = 0; i < kPlanPerThread; ++i) {
        const uint32_t b = b0 + i;
        if (b < B) {
            table[b] = run;
            if (b >= n_blocks)
                next[b] = 0u;
        }
        run += nk[i];
    }
}

__global__ void __launch_bounds__(kPlanThreads) plan_chunks_kernel(const uint32_t* counts, uint32_t B, uint32_t capacity,
                                                                    const uint32_t* reserved, uint32_t n_blocks,
                                                                    uint32_t* table, gf_out_desc* descs,
                                                                    const uint32_t* num_out, uint32_t* next,
                                                                    const uint32_t* status)
{
    if (ld_relaxed_u32(status) != 0u)
        return;
    const uint32_t R = *num_out;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < R || r < n_blocks; r += stride) {
        if (r < n_blocks)
            next[r] = 0u;
        if (r >= R)
            continue;
        uint32_t lo = 0, hi = B - 1u; // the last bin whose first chunk is at or before r
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1u) >> 1;
            if (table[mid] <= r)
                lo = mid;
            else
                hi = mid - 1u;
        }
        const uint32_t k = r - table[lo];
        const uint32_t chunk = __ldg(reserved + r);
        table[B + r] = chunk;
        descs[r].chunk_index = chunk;
        descs[r].fill = min(capacity, counts[lo] - k * capacity);
        descs[r].bin = lo;
    }
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
