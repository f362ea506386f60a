// Device-resident execution of a Flow (Tuning::deviceResident): the same graph, functors, keyed
// RNG streams and per-particle results as the host runner (runner.hpp), with the chunk pool on the
// device (gf_device_pool.cuh) and no host decision inside a wave.
//
// The run advances in waves. Every node owns an input list of chunks (id and fill) in device
// memory, in two sets: at a wave's start the host reads one small block (each list's chunk and
// particle counts, the status word) and then, for every node whose list holds chunks, enqueues the
// node's whole input as one batch on one stream; outputs are appended to the other set, which the
// next wave consumes. A transform forwards all its chunks to one node, so when that node comes later
// in the wave's node order (the runner orders every transform before its successor where the graph
// allows) the chunks join the successor's input of the same wave instead: a run of transforms and
// the node after them take one wave. The reference's runner (sched/GraphRunner.hpp:762-1171)
// instead dispatches batches of at most Q chunks and decides per batch on the host; both reach
// every particle with the same functor calls, since every draw is keyed by the particle
// (rng/ParticleRng.hpp:57-94).
//   source     wave 0: reserves ceil(n / C) chunks, generates ids 0..n-1 into them;
//   partition  tiles of 1024 particles from the list with the reservation of
//              outputChunkBound(particles, C, B) chunks from the device pool (the credit of
//              GraphRunner.hpp:1014-1037); one fused classify -> scan -> scatter launch that also
//              publishes the output descriptors; every output chunk appended to the list of the
//              node its port feeds, with the unused reservations returned and the input chunks
//              released: two launches, the tiles and reservation, then the cooperative
//              any-payload kernel of gf_fused_any.cuh (large batches) or the per-tile kernel of
//              gf_partition.cuh, whose finishing CTA also routes and settles;
//   transform  one launch: the functor applied in place and the chunks forwarded to the next node
//              (the reference's TransformKernel copies into a dense concatenation,
//              Execution.hpp:694-776; the particles and their order inside a chunk are the same);
//   sink       one launch: the functor over every particle and the chunks released.
// Pool: 2 (ceil(n / C) + sum of port counts + 2) + max ports + 16 chunks cover the chunks that hold
// particles at a wave boundary (full chunks and at most one partial chunk per port and producer)
// plus one batch's reservation. Exhaustion fails the run with GF_OVERFLOW (no waiting).
#pragma once

#include <algorithm>
#include <chrono>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "gf_device_pool.cuh"
#include "gf_fused_any.cuh"
#include "kernels.cuh"
#include "wave_order.hpp"

namespace graphflow {
namespace devflow {

inline constexpr std::uint32_t kNoList = 0xFFFFFFFFu;
inline constexpr std::uint32_t kTile = 1024u;

// Chunk lists: set s, list j at (s * N + j) * cap.
struct Lists {
    std::uint32_t* ids = nullptr;
    std::uint32_t* fills = nullptr;
    std::uint32_t* counts = nullptr;           // [2][N] chunks
    unsigned long long* particles = nullptr;   // [2][N]
    std::uint32_t N = 0u, cap = 0u;
    __host__ __device__ std::size_t at(std::uint32_t set, std::uint32_t j) const
    {
        return (static_cast<std::size_t>(set) * N + j) * cap;
    }
};

__device__ inline void appendChunk(const Lists& L, std::uint32_t set, std::uint32_t j, std::uint32_t id,
                                   std::uint32_t fill, std::uint32_t* status)
{
    if (j >= L.N) {
        gf::set_status(status, GF_INVALID);
        return;
    }
    const std::uint32_t pos = atomicAdd(&L.counts[set * L.N + j], 1u);
    if (pos >= L.cap) {
        gf::set_status(status, GF_OVERFLOW);
        return;
    }
    L.ids[L.at(set, j) + pos] = id;
    L.fills[L.at(set, j) + pos] = fill;
    atomicAdd(&L.particles[set * L.N + j], static_cast<unsigned long long>(fill));
}

// Zeroes the counters of list set `set` (kNoList: none) for its use as the next wave's output set.
// The first prep kernel of a wave runs it on the set the wave reads: the host has copied those
// counters before the wave's launches, and no kernel of the wave reads them on the device.
__device__ inline void clearSet(const Lists& L, std::uint32_t set)
{
    if (set >= 2u)
        return;
    for (std::uint32_t j = threadIdx.x; j < L.N; j += blockDim.x) {
        L.counts[set * L.N + j] = 0u;
        L.particles[set * L.N + j] = 0ull;
    }
}

// Source: particle i (id i) at slot i mod C of chunk chunk_of[i / C].
template <typename TFunctor, typename TView>
__global__ void __launch_bounds__(256)
    wave_source_kernel(TFunctor f, TView view, std::uint64_t seed_mixed, std::uint32_t purpose, std::uint64_t n,
                       const std::uint32_t* chunk_of, std::uint32_t num_chunks, std::uint32_t C, std::uint32_t* status)
{
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const std::uint32_t chunk = chunk_of[i / C];
        if (chunk >= num_chunks)
            continue; // a failed reservation: the status word already says so
        rng::Engine engine = rng::makeEngine(seed_mixed, i, 0u, purpose);
        Status st(status);
        auto payload = invokeWithContext(f, engine, st, i);
        view.store(static_cast<std::uint64_t>(chunk) * C + i % C, static_cast<typename TView::Payload>(payload));
    }
}

namespace { // internal linkage: every translation unit that runs a Flow has its own kernels

// The source's chunks (fills C, the last one the rest of n) into list `dst` of `set`.
__global__ void wave_source_list_kernel(const std::uint32_t* chunk_of, std::uint32_t k, std::uint64_t n,
                                        std::uint32_t C, Lists L, std::uint32_t set, std::uint32_t dst,
                                        std::uint32_t* status)
{
    for (std::uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < k; f += gridDim.x * blockDim.x) {
        const std::uint64_t left = n - static_cast<std::uint64_t>(f) * C;
        appendChunk(L, set, dst, chunk_of[f], static_cast<std::uint32_t>(left < C ? left : C), status);
    }
}

// Per-node kernels of a wave. Each folds a node's small steps into as few launches as stream order
// allows (a wave's tail is a few chunks per node, where every launch costs more than its work):
// the pool steps run in block 0 (pool_acquire_block / pool_settle_block), the list and tile steps
// in every block.

// tp tiles per list entry: entry f's tile j covers [j T, min(fill, (j + 1) T)) (empty past the fill).
__device__ inline void buildTiles(const std::uint32_t* ids, const std::uint32_t* fills, std::uint32_t k,
                                  std::uint32_t T, std::uint32_t tp, gf_tile* tiles)
{
    const std::uint32_t total = k * tp;
    for (std::uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const std::uint32_t f = t / tp, j = t - f * tp, off = j * T, fill = fills[f];
        tiles[t] = gf_tile{ids[f], off, fill > off ? (fill - off < T ? fill - off : T) : 0u};
    }
}

// Partition, before the partition kernel: its tiles; in block 0 the reservation of `bound` output
// chunks, the control block's three reset words (per-tile kernel) or the header of the
// cooperative kernel's scratch, and clearSet(clear).
__global__ void wave_partition_prep_kernel(const std::uint32_t* ids, const std::uint32_t* fills, std::uint32_t k,
                                           std::uint32_t T, std::uint32_t tp, gf_tile* tiles, gf::DevicePoolHdr* pool,
                                           std::uint32_t bound, std::uint32_t* reserved, gf::FusedCtl* ctl,
                                           gf::AnyCoopHdr* coop_hdr, Lists L, std::uint32_t clear,
                                           std::uint32_t* status)
{
    buildTiles(ids, fills, k, T, tp, tiles);
    if (blockIdx.x == 0) {
        if (ctl != nullptr && threadIdx.x < gf::kFusedCtlResetBytes / 4u)
            reinterpret_cast<std::uint32_t*>(ctl)[threadIdx.x] = 0u;
        if (coop_hdr != nullptr)
            for (std::uint32_t i = threadIdx.x; i < sizeof(gf::AnyCoopHdr) / 8u; i += blockDim.x)
                reinterpret_cast<unsigned long long*>(coop_hdr)[i] = 0ull;
        clearSet(L, clear);
        gf::pool_acquire_block(pool, bound, reserved, status);
    }
}

// The transform in one launch: block t runs tile t of the k entries (entry f = t / tp, particles
// [j T, min(fill, (j + 1) T)) of chunk ids[f], j = t - f tp), applying the functor in place (each
// particle back to its own slot, as transform_kernel with out_chunks = ids); block 0 runs
// clearSet(clear). Thread 0 of entry f's first tile forwards the entry to list `to` of set
// `to_set`: with base == kNoList appended (counters of to_set, the next wave's set), otherwise
// written at entry base + f of the list, whose count the host keeps (the successor runs later in
// the same wave). The successor reads the chunk in a later launch.
template <typename TFunctor, typename TView>
__global__ void __launch_bounds__(256)
    wave_transform_kernel(TFunctor f, TView view, std::uint64_t seed_mixed, std::uint32_t purpose,
                          const std::uint32_t* ids, const std::uint32_t* fills, std::uint32_t k, std::uint32_t C,
                          std::uint32_t T, std::uint32_t tp, std::uint64_t slots, Lists L, std::uint32_t to_set,
                          std::uint32_t to, std::uint32_t base, std::uint32_t clear, std::uint32_t* status)
{
    if (blockIdx.x == 0)
        clearSet(L, clear);
    for (std::uint32_t t = blockIdx.x; t < k * tp; t += gridDim.x) {
        const std::uint32_t e = t / tp, off = (t - e * tp) * T, fill = fills[e], chunk = ids[e];
        const std::uint32_t count = fill > off ? (fill - off < T ? fill - off : T) : 0u;
        if (off == 0u && threadIdx.x == 0u) {
            if (base == kNoList) {
                appendChunk(L, to_set, to, chunk, fill, status);
            } else {
                L.ids[L.at(to_set, to) + base + e] = chunk;
                L.fills[L.at(to_set, to) + base + e] = fill;
            }
        }
        const std::uint64_t in_base = static_cast<std::uint64_t>(chunk) * C + off;
        for (std::uint32_t i = threadIdx.x; i < count; i += blockDim.x) {
            if (in_base + i >= slots) {
                gf::set_status(status, GF_INVALID);
                continue;
            }
            auto p = view.load(in_base + i);
            rng::Engine engine = rng::engineFor(seed_mixed, p, purpose);
            Status st(status);
            applyTransform(f, engine, st, p);
            view.store(in_base + i, p);
        }
    }
}

// The sink in one launch: tiles as wave_transform_kernel, the functor over every particle; block 0
// runs clearSet(clear) and releases the k input chunks. Releasing them while other blocks still
// read them is safe in stream order: the next acquisition, which could hand them out again, comes
// after this launch.
template <typename TFunctor, typename TView>
__global__ void __launch_bounds__(256)
    wave_sink_kernel(TFunctor f, TView view, std::uint64_t seed_mixed, std::uint32_t purpose,
                     const std::uint32_t* ids, const std::uint32_t* fills, std::uint32_t k, std::uint32_t C,
                     std::uint32_t T, std::uint32_t tp, std::uint64_t slots, gf::DevicePoolHdr* pool, Lists L,
                     std::uint32_t clear, std::uint32_t* status)
{
    for (std::uint32_t t = blockIdx.x; t < k * tp; t += gridDim.x) {
        const std::uint32_t e = t / tp, off = (t - e * tp) * T, fill = fills[e];
        const std::uint32_t count = fill > off ? (fill - off < T ? fill - off : T) : 0u;
        const std::uint64_t in_base = static_cast<std::uint64_t>(ids[e]) * C + off;
        for (std::uint32_t i = threadIdx.x; i < count; i += blockDim.x) {
            if (in_base + i >= slots) {
                gf::set_status(status, GF_INVALID);
                continue;
            }
            const auto p = view.load(in_base + i);
            rng::Engine engine = rng::engineFor(seed_mixed, p, purpose);
            Status st(status);
            invokeWithContext(f, engine, st, p);
        }
    }
    if (blockIdx.x == 0) {
        clearSet(L, clear);
        gf::pool_settle_block(pool, nullptr, 0u, nullptr, 0u, ids, 1u, nullptr, k, status);
    }
}

// A partition batch's routing and settle, run by the partition kernel's finishing CTA after the
// output descriptors are published (the per-tile kernel's last CTA after its inline finish, the
// cooperative kernel's last CTA to finish): every output chunk appended to the list of the node
// its port feeds (route[bin]), the unused reservations returned and the k input chunks released
// (every CTA has read them by then).
struct WavePost {
    static constexpr bool kActive = true;
    const std::uint32_t* route = nullptr;
    std::uint32_t bins = 0u;
    Lists L;
    std::uint32_t set = 0u;
    gf::DevicePoolHdr* pool = nullptr;
    const std::uint32_t* reserved = nullptr;
    const std::uint32_t* ids = nullptr;
    std::uint32_t k = 0u;
    __device__ void operator()(const gf::InlineFinish& fin, std::uint32_t* status) const
    {
        const std::uint32_t n = *fin.num_out, m = n < fin.desc_cap ? n : fin.desc_cap;
        for (std::uint32_t f = threadIdx.x; f < m; f += blockDim.x) {
            const gf_out_desc d = fin.descs[f];
            if (d.bin >= bins || d.fill == 0u) {
                if (d.bin >= bins)
                    gf::set_status(status, GF_INVALID);
                continue;
            }
            appendChunk(L, set, route[d.bin], d.chunk_index, d.fill, status);
        }
        gf::pool_settle_block(pool, reserved, fin.desc_cap, fin.num_out, 0u, ids, 1u, nullptr, k, status);
    }
};

} // namespace

inline unsigned gridFor(std::uint64_t items, unsigned threads = 256u, unsigned cap = 4096u)
{
    const std::uint64_t g = (items + threads - 1u) / threads;
    return static_cast<unsigned>(std::max<std::uint64_t>(1u, std::min<std::uint64_t>(g, cap)));
}

// Buffers shared by every node of a run (one stream: a node's batch uses them and is done before
// the next node's batch starts).
struct WaveContext {
    cudaStream_t s = nullptr;
    gf::DevicePoolHdr* pool = nullptr;
    Lists L;
    std::uint32_t* status = nullptr;
    std::uint32_t C = 0u, T = kTile, tp = 1u;
    std::uint32_t numChunks = 0u;
    std::uint64_t slots = 0u;
    std::uint64_t seedMixed = 0u;
    gf_tile* tiles = nullptr;
    std::uint32_t* reserved = nullptr;
    std::uint32_t* totals = nullptr;
    unsigned long long* portChunks = nullptr;
    std::uint32_t maxK = 0u;
    gf::FusedCtl* ctl = nullptr;
    std::uint32_t* table = nullptr;
    gf_out_desc* descs = nullptr;
    std::uint32_t descCap = 0u;
    std::uint32_t* numOut = nullptr;
    // cooperative partitions (gf_fused_any.cuh) for batches of at least kCoopMinTiles tiles
    void* coopScratch = nullptr;
    std::uint64_t coopScratchBytes = 0u;
    std::uint32_t coopMaxCtas = 0u;
    int sms = 1;
    // the host's copy of the counts of the set the wave reads, and every node's position in the
    // wave's order: a transform whose successor comes later forwards into that set (same wave)
    std::uint32_t* waveCounts = nullptr;
    unsigned long long* waveParticles = nullptr;
    const std::uint32_t* order = nullptr;
    // the list set the wave's first prep kernel zeroes (clearSet), kNoList once one has
    std::uint32_t pendingClear = kNoList;
    std::uint32_t takeClearSet()
    {
        const std::uint32_t c = pendingClear;
        pendingClear = kNoList;
        return c;
    }
    std::uint64_t launches = 0u, partitionBatches = 0u, batches = 0u, sunk = 0u, coopBatches = 0u;
};

inline constexpr std::uint32_t kCoopMinTiles = 64u;

// One node's wave step. `routes` are the list indices its ports feed (device copy in routesDev).
class WaveNode {
public:
    virtual ~WaveNode() = default;
    // source only: generate n particles into reserved chunks, append them to list `to` of `set`
    virtual void generate(WaveContext&, std::uint64_t, std::uint32_t, std::uint32_t)
    {
        throw std::logic_error("graphflow: only a source generates");
    }
    // the node's whole input (k chunks, `particles` particles, list `self` of set `cur`) as one batch
    virtual void run(WaveContext& w, std::uint32_t self, std::uint32_t k, std::uint64_t particles,
                     std::uint32_t cur, std::uint32_t next, const std::vector<std::uint32_t>& routes,
                     const std::uint32_t* routesDev) = 0;
    virtual std::uint32_t bins() const { return 1u; }
    virtual void bind(std::uint32_t) {}
    // true when every input chunk goes on, unchanged in count, to routes[0] (a transform)
    virtual bool forwardsAll() const { return false; }
};

template <typename TStorage, typename TFunctor>
class SourceWave final : public WaveNode {
public:
    SourceWave(TStorage& st, TFunctor f, std::uint32_t purpose) : m_st(st), m_f(std::move(f)), m_purpose(purpose) {}
    void generate(WaveContext& w, std::uint64_t n, std::uint32_t set, std::uint32_t to) override
    {
        const std::uint32_t k = static_cast<std::uint32_t>((n + w.C - 1u) / w.C);
        // the reservation lands in this run's source list, which no route targets
        std::uint32_t* ids = w.L.ids + w.L.at(0u, m_self);
        gf::pool_acquire_kernel<<<1, gf::kPoolThreads, 0, w.s>>>(w.pool, k, ids, w.status);
        wave_source_kernel<<<gridFor(n, 256u, 148u * 16u), 256, 0, w.s>>>(m_f, m_st.view(), w.seedMixed, m_purpose,
                                                                        n, ids, w.numChunks, w.C, w.status);
        wave_source_list_kernel<<<gridFor(k), 256, 0, w.s>>>(ids, k, n, w.C, w.L, set, to, w.status);
        cuda::check(cudaGetLastError(), "device-resident source launch");
        w.launches += 3u;
        ++w.batches;
    }
    void run(WaveContext&, std::uint32_t, std::uint32_t, std::uint64_t, std::uint32_t, std::uint32_t,
             const std::vector<std::uint32_t>&, const std::uint32_t*) override
    {
        throw std::logic_error("graphflow: a source has no input");
    }
    void bind(std::uint32_t self) override { m_self = self; }

private:
    TStorage& m_st;
    TFunctor m_f;
    std::uint32_t m_purpose;
    std::uint32_t m_self = 0u;
};

template <typename TStorage, typename TFunctor>
class TransformWave final : public WaveNode {
public:
    TransformWave(TStorage& st, TFunctor f, std::uint32_t purpose) : m_st(st), m_f(std::move(f)), m_purpose(purpose) {}
    bool forwardsAll() const override { return true; }
    void run(WaveContext& w, std::uint32_t self, std::uint32_t k, std::uint64_t particles, std::uint32_t cur,
             std::uint32_t next, const std::vector<std::uint32_t>& routes, const std::uint32_t*) override
    {
        const std::uint32_t* ids = w.L.ids + w.L.at(cur, self);
        const std::uint32_t* fills = w.L.fills + w.L.at(cur, self);
        const std::uint32_t nt = k * w.tp;
        const std::uint32_t to = routes[0];
        std::uint32_t toSet = next, base = kNoList;
        if (w.waveCounts != nullptr && to < w.L.N && w.order[to] > w.order[self]) {
            // the successor runs later in this wave: its input list of this wave grows by k chunks
            base = w.waveCounts[to];
            if (static_cast<std::uint64_t>(base) + k > w.L.cap)
                throw BatchError("graphflow: device-resident list overflow");
            toSet = cur;
            w.waveCounts[to] = base + k;
            w.waveParticles[to] += particles;
        }
        wave_transform_kernel<<<nt, 256, 0, w.s>>>(m_f, m_st.view(), w.seedMixed, m_purpose, ids, fills, k, w.C, w.T,
                                                   w.tp, w.slots, w.L, toSet, to, base, w.takeClearSet(), w.status);
        cuda::check(cudaGetLastError(), "device-resident transform launch");
        ++w.launches;
        ++w.batches;
    }

private:
    TStorage& m_st;
    TFunctor m_f;
    std::uint32_t m_purpose;
};

template <typename TStorage, typename TFunctor>
class SinkWave final : public WaveNode {
public:
    SinkWave(TStorage& st, TFunctor f, std::uint32_t purpose) : m_st(st), m_f(std::move(f)), m_purpose(purpose) {}
    void run(WaveContext& w, std::uint32_t self, std::uint32_t k, std::uint64_t particles, std::uint32_t cur,
             std::uint32_t, const std::vector<std::uint32_t>&, const std::uint32_t*) override
    {
        const std::uint32_t* ids = w.L.ids + w.L.at(cur, self);
        const std::uint32_t* fills = w.L.fills + w.L.at(cur, self);
        const std::uint32_t nt = k * w.tp;
        wave_sink_kernel<<<nt, 256, 0, w.s>>>(m_f, m_st.view(), w.seedMixed, m_purpose, ids, fills, k, w.C, w.T, w.tp,
                                              w.slots, w.pool, w.L, w.takeClearSet(), w.status);
        cuda::check(cudaGetLastError(), "device-resident sink launch");
        ++w.launches;
        w.sunk += particles;
        ++w.batches;
    }

private:
    TStorage& m_st;
    TFunctor m_f;
    std::uint32_t m_purpose;
};

template <typename TStorage, typename TClassifier, typename TUpdate, typename TBin>
class PartitionWave final : public WaveNode {
    using View = typename TStorage::View;
    using P = typename TStorage::Payload;
    using Acc = ViewAccess<View>;
    using Cls = ClassifyAdapter<TClassifier, P>;
    using Upd = UpdateAdapter<TUpdate, TBin, P>;
    using Shape = gf::TileShape<256, 4, 2>; // 1024-particle tiles, as PartitionStage
    // the cooperative kernel: the same tiles; payloads of up to 32 bytes at three CTAs per SM (at
    // most 85 registers per thread), wider ones (the FP64 photon) at two, which keeps them unspilled
    using CoopShape = std::conditional_t<(sizeof(P) <= 32u), gf::TileShape<256, 4, 3>, gf::TileShape<256, 4, 2>>;
    static_assert(Shape::kTile == kTile && CoopShape::kTile == kTile, "tile size");

public:
    PartitionWave(TStorage& st, TClassifier cls, TUpdate upd, std::uint32_t bins, std::uint32_t purpose)
        : m_st(st), m_cls(std::move(cls)), m_upd(std::move(upd)), m_bins(bins), m_purpose(purpose)
    {
        m_smem = smemBytes(bins);
        int dev = 0, limit = 0;
        cuda::check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda::check(cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "smem limit");
        cudaFuncAttributes fa{}; // the finishing CTA's settle adds a few bytes of static shared memory
        cuda::check(cudaFuncGetAttributes(&fa, gf::fused_partition_kernel<Shape, Acc, Cls, Upd, WavePost>),
                    "device-resident partition attributes");
        if (m_smem + fa.sharedSizeBytes > static_cast<std::size_t>(limit))
            throw std::invalid_argument("graphflow: deviceResident runs dense fused partitions only; " +
                                        std::to_string(bins) + " ports do not fit one block's shared memory");
        cuda::check(cudaFuncSetAttribute(gf::fused_partition_kernel<Shape, Acc, Cls, Upd, WavePost>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(m_smem)),
                    "device-resident partition attribute");
    }
    static std::size_t smemBytes(std::uint32_t bins)
    {
        return sizeof(P) * Shape::kTile + 4u * Shape::kTile + 4u * Shape::kWarps * bins + 4u * bins * 6u +
               4u * (2u * Shape::kThreads + Shape::kWarps + 8u);
    }
    std::uint32_t bins() const override { return m_bins; }
    void run(WaveContext& w, std::uint32_t self, std::uint32_t k, std::uint64_t particles, std::uint32_t cur,
             std::uint32_t next, const std::vector<std::uint32_t>&, const std::uint32_t* routesDev) override
    {
        const std::uint32_t* ids = w.L.ids + w.L.at(cur, self);
        const std::uint32_t* fills = w.L.fills + w.L.at(cur, self);
        const std::uint32_t nt = k * w.tp;
        const std::uint64_t b64 = checkedOutputChunkBound(particles, w.C, m_bins);
        if (b64 > w.descCap)
            throw BatchError("graphflow: deviceResident batch needs more output chunks than the run reserved");
        const std::uint32_t bound = static_cast<std::uint32_t>(b64);
        const bool coop =
            w.coopScratch != nullptr && m_bins <= gf::kAnyCoopMaxBins && nt >= kCoopMinTiles;
        wave_partition_prep_kernel<<<gridFor(nt), 256, 0, w.s>>>(
            ids, fills, k, w.T, w.tp, w.tiles, w.pool, bound, w.reserved, coop ? nullptr : w.ctl,
            coop ? static_cast<gf::AnyCoopHdr*>(w.coopScratch) : nullptr, w.L, w.takeClearSet(), w.status);
        const Acc acc{m_st.view()};
        const Cls cls{m_cls, w.seedMixed, m_purpose, w.status};
        const Upd upd{m_upd, m_purpose + 1u, w.status};
        const gf::InlineFinish fin{w.table, w.descs, bound, w.numOut};
        // the partition kernel's finishing CTA routes the outputs and settles the pool
        const WavePost post{routesDev, m_bins, w.L, next, w.pool, w.reserved, ids, k};
        if (coop) {
            // a large batch: count, one grid barrier, plan, scatter (no per-tile look-back); the
            // prep kernel zeroed the scratch header
            cuda::check(gf::launch_fused_any_coop<CoopShape>(w.s, acc, cls, upd, w.seedMixed, w.C, w.slots, w.tiles, nt,
                                                             m_bins, w.reserved, bound, w.totals, w.coopScratch,
                                                             w.coopScratchBytes, w.coopMaxCtas, w.status, fin, w.sms,
                                                             post, false),
                        "device-resident cooperative partition launch");
            ++w.coopBatches;
        } else {
            auto* desc = reinterpret_cast<unsigned long long*>(w.ctl + 1); // reset words zeroed by the prep kernel
            // the launch's last CTA builds the table and the output descriptors
            gf::fused_partition_kernel<Shape, Acc, Cls, Upd, WavePost><<<nt, Shape::kThreads, m_smem, w.s>>>(
                acc, cls, upd, w.seedMixed, w.C, gf::FastDiv(w.C), w.slots, w.tiles, nt, m_bins, w.reserved, bound,
                w.totals, w.portChunks, w.maxK, w.ctl, desc, w.status, fin, post);
        }
        cuda::check(cudaGetLastError(), "device-resident partition launch");
        w.launches += 2u;
        ++w.partitionBatches;
        ++w.batches;
    }

private:
    TStorage& m_st;
    TClassifier m_cls;
    TUpdate m_upd;
    std::uint32_t m_bins, m_purpose;
    std::size_t m_smem = 0u;
};

} // namespace devflow
} // namespace graphflow
