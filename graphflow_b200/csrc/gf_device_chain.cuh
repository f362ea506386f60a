// The dense classify chain (Generate -> 1..4 partition nodes -> sink, examples/dense_chain.cuh's
// graph) run entirely on the device: one stream, no host round trip between nodes, chunks from a
// device-resident pool (gf_device_pool.cuh). Every node runs as one fused partition launch over all
// of its input (the whole-batch form of PartitionStage::planAndScatter, flow/Execution.hpp:
// 2363-2642), so the host never reads a count before the next launch:
//   source    the pool reserves ceil(n / C) chunks; ids 0..n-1 and their keys fill them in order;
//   node i    tiles from the previous stage's published chunks (two tiles of at most 4096 records
//             per chunk; a node's input has at most outputChunkBound chunks, so the tile count is
//             known on the host and the entries past the real chunks are empty tiles); the pool
//             reserves outputChunkBound(n, C, B); the fused kernel (gf_partition.cuh) partitions,
//             plans and publishes the output chunks in its last CTA; the settle step returns the
//             unused reservations and releases the node's input chunks;
//   sink      every id in the last node's published chunks records its port; the chunks go back.
// Pool size: a node holds its input (at most max(ceil(n / C), bound) chunks) and its reservation,
// so S = max(ceil(n / C), bound) + bound chunks serve a chain of any length.
#pragma once

#include <algorithm>

#include "../examples/dense_chain.cuh"
#include "gf_device_pool.cuh"
#include "gf_fused_any.cuh"
#include "gf_partition.cuh"

namespace gf {
namespace { // internal linkage: see gf_partition.cuh

constexpr std::uint32_t kChainCapacity = 8192u;
constexpr std::uint32_t kChainTile = 4096u;

struct KeyIdColumns { // {u32 id, u32 key} in two pool columns; a batch reads and writes distinct chunks
    using Payload = graphflow::dense::KeyRecord;
    std::uint32_t* id;
    std::uint32_t* key;
    GF_D Payload load(std::uint64_t s) const { return Payload{id[s], key[s]}; }
    GF_D void store(std::uint64_t s, const Payload& p) const
    {
        id[s] = p.id;
        key[s] = p.key;
    }
};

struct ShiftPort { // node i: port = (key >> 8 i) mod B (dense_chain.cuh's PortOfKey)
    std::uint32_t shift;
    FastDiv fd;
    GF_D std::uint32_t operator()(const graphflow::dense::KeyRecord& r) const { return fd.mod(r.key >> shift); }
};

using ChainShape = TileShape<256, 16, 3>;
static_assert(ChainShape::kTile == kChainTile && kChainCapacity == 2u * kChainTile, "two tiles per chunk");

// Source: record i = {i, key_i} at slot i mod C of chunk chunk_of[i / C] (a chunk id the pool
// did not grant, numChunks or above, is skipped; the failed reservation is in the status word).
__global__ void chain_source_kernel(std::uint64_t seedMixed, int dist, std::uint32_t bins, const double* cdf,
                                    std::uint64_t n, const std::uint32_t* chunk_of, std::uint32_t numChunks,
                                    std::uint32_t* id, std::uint32_t* key)
{
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const std::uint32_t chunk = chunk_of[i / kChainCapacity];
        if (chunk >= numChunks)
            continue;
        const std::uint64_t s = static_cast<std::uint64_t>(chunk) * kChainCapacity + i % kChainCapacity;
        id[s] = static_cast<std::uint32_t>(i);
        key[s] = synthetic_key(dist, seedMixed, i, bins, cdf);
    }
}

// Two tiles per chunk: the source's chunks (chunk_of, the last one partly filled), or a node's
// published output chunks (descs[0 .. *numOut)); entries past them are empty tiles.
__global__ void chain_tiles_kernel(std::uint64_t n, std::uint32_t nChunks, const std::uint32_t* chunk_of,
                                   const gf_out_desc* descs, const std::uint32_t* numOut, gf_tile* tiles)
{
    for (std::uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < nChunks; f += gridDim.x * blockDim.x) {
        std::uint32_t chunk = 0, fill = 0;
        if (descs == nullptr) {
            chunk = chunk_of[f];
            const std::uint64_t left = n - static_cast<std::uint64_t>(f) * kChainCapacity;
            fill = static_cast<std::uint32_t>(left < kChainCapacity ? left : kChainCapacity);
        } else if (f < *numOut) {
            chunk = descs[f].chunk_index;
            fill = descs[f].fill;
        }
        tiles[2u * f] = gf_tile{chunk, 0u, fill < kChainTile ? fill : kChainTile};
        tiles[2u * f + 1u] = gf_tile{chunk, kChainTile, fill > kChainTile ? fill - kChainTile : 0u};
    }
}

// Sink: each published output chunk of the last node records its port for every id in it and
// counts the records it saw (a chunk id numChunks or above, from a failed reservation, is skipped).
// The ports (below 255) go to a byte per id: the ids arrive in no order, and N bytes fit the
// 126 MB L2 at N = 1e8 where N words do not, so the scattered writes merge in L2 instead of each
// costing a DRAM sector; chain_expand_kernel widens them afterwards with streaming stores.
__global__ void chain_sink_kernel(const gf_out_desc* descs, const std::uint32_t* numOut, std::uint32_t numChunks,
                                  const std::uint32_t* id, std::uint8_t* port8, std::uint64_t n,
                                  unsigned long long* sunk)
{
    for (std::uint32_t f = blockIdx.x; f < *numOut; f += gridDim.x) {
        const gf_out_desc d = descs[f];
        if (d.chunk_index >= numChunks || d.fill > kChainCapacity)
            continue;
        const std::uint64_t base = static_cast<std::uint64_t>(d.chunk_index) * kChainCapacity;
        for (std::uint32_t i = threadIdx.x; i < d.fill; i += blockDim.x) {
            const std::uint32_t who = id[base + i];
            if (who < n)
                port8[who] = static_cast<std::uint8_t>(d.bin);
        }
        if (threadIdx.x == 0 && sunk != nullptr)
            atomicAdd(sunk, static_cast<unsigned long long>(d.fill));
    }
}

// portOf[i] = port8[i], 0xFF (no port recorded) widened to 0xFFFFFFFF; four ids per thread step.
__global__ void chain_expand_kernel(const std::uint8_t* port8, std::uint32_t* portOf, std::uint64_t n)
{
    auto widen = [](std::uint32_t b) { return b == 0xFFu ? 0xFFFFFFFFu : b; };
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    const std::uint64_t n4 = n / 4u;
    for (std::uint64_t q = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < n4; q += stride) {
        const std::uint32_t v = reinterpret_cast<const std::uint32_t*>(port8)[q];
        reinterpret_cast<uint4*>(portOf)[q] =
            make_uint4(widen(v & 0xFFu), widen((v >> 8) & 0xFFu), widen((v >> 16) & 0xFFu), widen(v >> 24));
    }
    for (std::uint64_t i = 4u * n4 + static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += stride)
        portOf[i] = widen(port8[i]);
}

// Byte offsets of one chain run's buffers inside one device block (every buffer 256-byte aligned).
struct DeviceChainLayout {
    std::uint64_t n;
    std::uint32_t bins, nodes;
    std::uint64_t nIn, bound, chunks, slots, tiles, maxK;
    std::uint64_t pool, id, key, tile, srcIds, reserved, scratch, totals, portChunks, table, descs[2], numOut,
        sunk, portOf, port8, coop, coopBytes, total;
    std::uint32_t coopCtas;
    // coop_ctas: rows of the cooperative kernel's scratch (0: every node runs the per-tile kernel)
    DeviceChainLayout(std::uint64_t n_, std::uint32_t bins_, std::uint32_t nodes_, std::uint64_t bound_,
                      std::uint32_t coop_ctas = 0u)
        : n(n_), bins(bins_), nodes(nodes_), coopCtas(coop_ctas)
    {
        nIn = (n + kChainCapacity - 1u) / kChainCapacity;
        bound = bound_;
        chunks = std::max(nIn, bound) + bound;
        slots = chunks * kChainCapacity;
        tiles = 2u * std::max(nIn, bound);
        maxK = std::max<std::uint64_t>(nIn, 1u);
        auto up = [](std::uint64_t v) { return (v + 255u) & ~std::uint64_t(255u); };
        std::uint64_t o = 0;
        auto take = [&](std::uint64_t& at, std::uint64_t bytes) {
            at = o;
            o += up(bytes);
        };
        take(pool, device_pool_bytes(static_cast<std::uint32_t>(chunks)));
        take(id, slots * 4u);
        take(key, slots * 4u);
        take(tile, tiles * sizeof(gf_tile));
        take(srcIds, std::max<std::uint64_t>(nIn, 1u) * 4u);
        take(reserved, std::max<std::uint64_t>(bound, 1u) * 4u);
        take(scratch, 64u + tiles * bins * 8u);
        take(totals, static_cast<std::uint64_t>(nodes) * bins * 4u);
        take(portChunks, bins * maxK * 8u);
        take(table, (bins + bound) * 4u);
        take(descs[0], std::max<std::uint64_t>(bound, 1u) * sizeof(gf_out_desc));
        take(descs[1], std::max<std::uint64_t>(bound, 1u) * sizeof(gf_out_desc));
        take(numOut, 256u);
        take(sunk, 256u);
        take(portOf, std::max<std::uint64_t>(n, 1u) * 4u);
        take(port8, std::max<std::uint64_t>(n, 1u));
        coopBytes = coopCtas ? any_coop_scratch_bytes(static_cast<std::uint32_t>(tiles), kChainTile, coopCtas) : 0u;
        take(coop, coopBytes);
        total = o;
    }
};

// Enqueues the whole chain on `s`: ports into portOf[n], node i's per-port totals into
// totals[i * bins ..], failures into *status. Returns the number of kernel launches.
inline std::uint32_t enqueueDeviceChain(cudaStream_t s, char* base, const DeviceChainLayout& L, int dist,
                                        const double* cdf, std::uint64_t seed, std::uint32_t* status,
                                        std::uint32_t sms)
{
    auto P = [&](std::uint64_t off) { return base + off; };
    auto* pool = reinterpret_cast<DevicePoolHdr*>(P(L.pool));
    auto* id = reinterpret_cast<std::uint32_t*>(P(L.id));
    auto* key = reinterpret_cast<std::uint32_t*>(P(L.key));
    auto* tiles = reinterpret_cast<gf_tile*>(P(L.tile));
    auto* srcIds = reinterpret_cast<std::uint32_t*>(P(L.srcIds));
    auto* reserved = reinterpret_cast<std::uint32_t*>(P(L.reserved));
    auto* ctl = reinterpret_cast<FusedCtl*>(P(L.scratch));
    auto* desc = reinterpret_cast<unsigned long long*>(ctl + 1);
    auto* totals = reinterpret_cast<std::uint32_t*>(P(L.totals));
    auto* portChunks = reinterpret_cast<unsigned long long*>(P(L.portChunks));
    auto* table = reinterpret_cast<std::uint32_t*>(P(L.table));
    gf_out_desc* descs[2] = {reinterpret_cast<gf_out_desc*>(P(L.descs[0])),
                             reinterpret_cast<gf_out_desc*>(P(L.descs[1]))};
    auto* numOut = reinterpret_cast<std::uint32_t*>(P(L.numOut)); // [2]
    auto* sunk = reinterpret_cast<unsigned long long*>(P(L.sunk));
    auto* portOf = reinterpret_cast<std::uint32_t*>(P(L.portOf));
    const std::uint32_t bins = L.bins;
    std::uint32_t launches = 0;
    auto check = [](cudaError_t e, const char* what) { graphflow::cuda::check(e, what); };
    const unsigned g = static_cast<unsigned>(std::min<std::uint64_t>((std::max<std::uint64_t>(L.n, 1u) + 255u) / 256u,
                                                                     sms * 8u));
    pool_init_kernel<<<static_cast<unsigned>(std::min<std::uint64_t>((L.chunks + 1023u) / 1024u + 1u, sms)),
                       kPoolThreads, 0, s>>>(pool, static_cast<std::uint32_t>(L.chunks));
    check(cudaMemsetAsync(P(L.port8), 0xFF, std::max<std::uint64_t>(L.n, 1u), s), "memset");
    launches += 1u;
    // A fresh control block restarts the launch epochs at 1, so epoch-tagged look-back descriptors
    // and chunk claims left in this block by an earlier run are cleared too (tag 0 never matches).
    check(cudaMemsetAsync(ctl, 0, 64u + L.tiles * bins * 8u, s), "memset");
    check(cudaMemsetAsync(portChunks, 0, bins * L.maxK * 8u, s), "memset");
    check(cudaMemsetAsync(numOut, 0, 256u, s), "memset");
    check(cudaMemsetAsync(sunk, 0, 256u, s), "memset");
    // source
    pool_acquire_kernel<<<1, kPoolThreads, 0, s>>>(pool, static_cast<std::uint32_t>(L.nIn), srcIds, status);
    chain_source_kernel<<<g, 256, 0, s>>>(mix64(seed), dist, bins, cdf, L.n, srcIds,
                                          static_cast<std::uint32_t>(L.chunks), id, key);
    launches += 2u;

    auto kernel = fused_partition_kernel<ChainShape, KeyIdColumns, ShiftPort, NoUpdate>;
    constexpr int W = ChainShape::kWarps;
    const std::size_t smem = sizeof(graphflow::dense::KeyRecord) * ChainShape::kTile + 4u * ChainShape::kTile +
                             4u * W * bins + 4u * bins * 6u + 4u * (W + 2u) + 16u +
                             4u * (4u + 2u * ChainShape::kThreads);
    check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
          "chain partition attribute");
    constexpr int FT = 1024;
    const std::size_t fsmem = sizeof(std::uint32_t) * (4096u * 2u + FT / 32 + 1);
    check(cudaFuncSetAttribute(fused_finish_kernel<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(fsmem)),
          "finish attribute");
    const FastDiv fdc(kChainCapacity);
    const KeyIdColumns cols{id, key};
    const std::uint32_t bound = static_cast<std::uint32_t>(L.bound);
    for (std::uint32_t node = 0; node < L.nodes; ++node) {
        const bool first = node == 0u;
        const gf_out_desc* in = first ? nullptr : descs[(node - 1u) & 1u];
        const std::uint32_t* inCount = first ? nullptr : numOut + ((node - 1u) & 1u);
        gf_out_desc* out = descs[node & 1u];
        std::uint32_t* outCount = numOut + (node & 1u);
        const std::uint32_t nChunks = static_cast<std::uint32_t>(first ? L.nIn : L.bound);
        const std::uint32_t nTiles = 2u * nChunks;
        chain_tiles_kernel<<<(nChunks + 255u) / 256u + 1u, 256, 0, s>>>(L.n, nChunks, srcIds, in, inCount, tiles);
        pool_acquire_kernel<<<1, kPoolThreads, 0, s>>>(pool, bound, reserved, status);
        std::uint32_t* nodeTotals = totals + static_cast<std::size_t>(node) * bins;
        if (nTiles != 0u && L.coopBytes != 0u && nTiles >= 64u && bins <= kAnyCoopMaxBins) {
            // count, one grid barrier, plan, scatter over the node's whole input
            check(launch_fused_any_coop<ChainShape>(s, cols, ShiftPort{8u * node, FastDiv(bins)}, NoUpdate{}, 0u,
                                                    kChainCapacity, L.slots, tiles, nTiles, bins, reserved, bound,
                                                    nodeTotals, P(L.coop), L.coopBytes, L.coopCtas, status,
                                                    InlineFinish{table, out, bound, outCount}, static_cast<int>(sms)),
                  "device chain cooperative partition");
        } else if (nTiles != 0u) {
            check(cudaMemsetAsync(ctl, 0, kFusedCtlResetBytes, s), "memset");
            // the last CTA builds this node's table and descriptors (no separate finish launch)
            kernel<<<nTiles, ChainShape::kThreads, smem, s>>>(
                cols, ShiftPort{8u * node, FastDiv(bins)}, NoUpdate{}, 0u, kChainCapacity, fdc, L.slots, tiles, nTiles,
                bins, reserved, bound, nodeTotals, portChunks, static_cast<std::uint32_t>(L.maxK), ctl, desc, status,
                InlineFinish{table, out, bound, outCount}, NoPost{});
        } else {
            check(cudaMemsetAsync(nodeTotals, 0, bins * 4u, s), "memset");
            fused_finish_kernel<FT><<<1, FT, fsmem, s>>>(nodeTotals, portChunks, bins, kChainCapacity, fdc,
                                                          static_cast<std::uint32_t>(L.maxK), ctl, table, out, bound,
                                                          outCount, status);
        }
        // unused reservations back, then this node's input chunks released
        pool_settle_kernel<<<1, kPoolThreads, 0, s>>>(pool, reserved, bound, outCount, 0u,
                                                      first ? srcIds : &in->chunk_index, first ? 1u : 3u, inCount,
                                                      static_cast<std::uint32_t>(L.nIn), status);
        launches += 4u;
    }
    const gf_out_desc* last = descs[(L.nodes - 1u) & 1u];
    const std::uint32_t* lastCount = numOut + ((L.nodes - 1u) & 1u);
    chain_sink_kernel<<<static_cast<unsigned>(std::min<std::uint64_t>(std::max<std::uint64_t>(L.bound, 1u), 4096u)),
                        256, 0, s>>>(last, lastCount, static_cast<std::uint32_t>(L.chunks), id,
                                     reinterpret_cast<std::uint8_t*>(P(L.port8)), L.n, sunk);
    chain_expand_kernel<<<g, 256, 0, s>>>(reinterpret_cast<const std::uint8_t*>(P(L.port8)), portOf, L.n);
    pool_settle_kernel<<<1, kPoolThreads, 0, s>>>(pool, nullptr, 0u, nullptr, 0u, &last->chunk_index, 3u, lastCount,
                                                  0u, status);
    launches += 3u;
    check(cudaGetLastError(), "device chain launch");
    return launches;
}

} // namespace
} // namespace gf
