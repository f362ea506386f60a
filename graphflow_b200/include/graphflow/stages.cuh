// Typed execution stages of the C++ front end. Each stage owns its per-batch device buffers and
// pinned host mirrors and exposes the hook protocol of the reference's StageBase
// (flow/Execution.hpp:1538-1561): launch -> [advance]* -> finish | abort.
//
//   SourceStage     flow/Execution.hpp:1582-1690   one chunk per batch, ids firstId + i
//   TransformStage  flow/Execution.hpp:1692-2258   out-of-place, dense output concatenation
//   PartitionStage  flow/Execution.hpp:2263-2772   classify -> plan -> scatter -> finalise, or the
//                                                  B200 fused classify->scan->scatter form
//   SinkStage       flow/Execution.hpp:2776-...    consumes the batch
#pragma once

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "gf_hash.cuh"
#include "kernels.cuh"
#include "stage.hpp"
#include "storage.cuh"

namespace graphflow {

namespace detail {

inline std::vector<MoveTile> moveTiles(const Batch& b, std::uint32_t tile)
{
    std::vector<MoveTile> out;
    std::uint32_t pos = 0;
    for (const auto& c : b.chunks)
        for (std::uint32_t off = 0; off < c.fill; off += tile) {
            const std::uint32_t n = c.fill - off < tile ? c.fill - off : tile;
            out.push_back(MoveTile{c.handle.index, off, n, pos});
            pos += n;
        }
    return out;
}

template <typename T>
struct Staged {
    cuda::Buffer<T> dev;
    cuda::HostBuffer<T> host;
    explicit Staged(std::size_t n = 0) : dev(n ? n : 1), host(n ? n : 1) {}
    void upload(cudaStream_t s, std::size_t n)
    {
        if (n)
            cuda::check(cudaMemcpyAsync(dev.data(), host.data(), n * sizeof(T), cudaMemcpyHostToDevice, s), "H2D");
    }
    void download(cudaStream_t s, std::size_t n)
    {
        if (n)
            cuda::check(cudaMemcpyAsync(host.data(), dev.data(), n * sizeof(T), cudaMemcpyDeviceToHost, s), "D2H");
    }
};

// A stage's device status word: zeroed once, written by a kernel only on a failure, so it is reset
// before a launch only after a batch has reported one (a failure normally ends the run).
struct StatusWord {
    Staged<std::uint32_t> w{1};
    bool dirty = false;
    StatusWord() { cuda::check(cudaMemset(w.dev.data(), 0, 4), "memset"); }
    std::uint32_t* dev() const { return w.dev.data(); }
    void prepare(cudaStream_t s)
    {
        if (dirty)
            cuda::check(cudaMemsetAsync(w.dev.data(), 0, 4, s), "memset");
        dirty = false;
    }
    void download(cudaStream_t s) { w.download(s, 1); }
    std::uint32_t read()
    {
        const std::uint32_t v = w.host[0];
        dirty = dirty || v != 0u;
        return v;
    }
};

// A front-end stage's host-polled completion record (Completion in kernels.cuh): [0] sequence,
// [1] status in mapped pinned memory, and the device counter the kernel's last CTA is elected by.
struct CompletionRecord {
    cuda::HostBuffer<std::uint32_t> rec{2};
    cuda::Buffer<std::uint32_t> ctas{1};
    std::uint32_t* recDev = nullptr;
    std::uint32_t seq = 0u;
    CompletionRecord()
    {
        rec.data()[0] = rec.data()[1] = 0u;
        cuda::check(cudaMemset(ctas.data(), 0, 4u), "memset");
        recDev = cuda::mappedDevicePointer(rec.data());
    }
    // the next launch's completion
    Completion arm()
    {
        ++seq;
        return Completion{ctas.data(), recDev, seq};
    }
    // a launch with nothing to run is complete at once
    void completeOnHost()
    {
        rec.data()[1] = 0u;
        reinterpret_cast<volatile std::uint32_t*>(rec.data())[0] = seq;
    }
    bool done() const
    {
        const bool d = reinterpret_cast<const volatile std::uint32_t*>(rec.data())[0] == seq;
        if (d)
            std::atomic_thread_fence(std::memory_order_acquire);
        return d;
    }
    std::uint32_t status() const { return rec.data()[1]; }
};

inline void checkStatusWord(std::uint32_t w, const char* stage)
{
    if (w != 0u)
        throw BatchError(std::string(stage) + ": device status reports " + statusCodeName(decodeStatus(w)) +
                         " (code " + std::to_string(w) + ")");
}

} // namespace detail

template <typename TStorage, typename TFunctor>
class SourceStage final : public Stage {
public:
    SourceStage(TStorage& st, const Config& c, TFunctor f, std::uint32_t purpose)
        : m_st(st), m_f(std::move(f)), m_seed(gf::mix64(c.seed)), m_purpose(purpose)
    {
    }
    std::uint32_t launch(cudaStream_t s, const Batch& b) override
    {
        if (b.chunks.size() != 1u)
            throw BatchError("source: a source batch is exactly one chunk");
        const auto& c = b.chunks[0];
        const Completion done = m_done.arm();
        const unsigned blocks = (c.fill + 255u) / 256u;
        if (blocks)
            source_kernel<<<blocks, 256, 0, s>>>(m_f, m_st.view(), m_seed, m_purpose, b.firstId,
                                                  m_st.base(c.handle), c.fill, m_status.dev(), done);
        else
            m_done.completeOnHost();
        cuda::check(cudaGetLastError(), "source launch");
        ++m_launches;
        return 0u;
    }
    bool pollsCompletion() const override { return true; }
    bool completed() const override { return m_done.done(); }
    bool advance(cudaStream_t, const Batch&, std::uint32_t& allocated) override
    {
        allocated = 0u;
        detail::checkStatusWord(m_done.status(), "source");
        return false;
    }
    void finish(const Batch& b, std::vector<ChunkDescriptor>& outputs) override
    {
        outputs.push_back(ChunkDescriptor{b.chunks[0].handle, b.chunks[0].fill, 0u});
    }
    void abort() override {}

private:
    TStorage& m_st;
    TFunctor m_f;
    std::uint64_t m_seed;
    std::uint32_t m_purpose;
    detail::StatusWord m_status;
    detail::CompletionRecord m_done;
};

template <typename TStorage, typename TFunctor>
class TransformStage final : public Stage {
public:
    TransformStage(TStorage& st, const Config& c, TFunctor f, std::uint32_t purpose)
        : m_st(st), m_f(std::move(f)), m_seed(gf::mix64(c.seed)), m_purpose(purpose), m_tile(1024u),
          m_tileCap(static_cast<std::uint32_t>(c.batchChunks) * ((c.chunkCapacity + 1023u) / 1024u)),
          m_io(4u * m_tileCap + c.batchChunks) // mapped: [tiles (4 words each) | output chunk indices]
    {
        static_assert(sizeof(MoveTile) == 16, "packed layout");
        m_ioDev = cuda::mappedDevicePointer(m_io.data());
    }
    std::uint32_t launch(cudaStream_t s, const Batch& b) override
    {
        const auto tiles = detail::moveTiles(b, m_tile);
        if (tiles.size() > m_tileCap)
            throw BatchError("transform: tile capacity exceeded");
        const std::uint64_t n = b.particles();
        const std::uint32_t C = m_st.chunkCapacity();
        const std::uint32_t r = static_cast<std::uint32_t>((n + C - 1u) / C);
        m_pending.clear();
        for (std::uint32_t k = 0; k < r; ++k) {
            const ChunkHandle h = m_st.ledger().acquire();
            m_io.data()[4u * m_tileCap + k] = h.index;
            const std::uint64_t left = n - static_cast<std::uint64_t>(k) * C;
            m_pending.push_back(ChunkDescriptor{h, static_cast<std::uint32_t>(left < C ? left : C), 0u});
        }
        if (!tiles.empty())
            std::memcpy(m_io.data(), tiles.data(), sizeof(MoveTile) * tiles.size());
        // the kernel reads the tiles and output chunk indices from mapped memory
        const Completion done = m_done.arm();
        auto* dtiles = reinterpret_cast<const MoveTile*>(m_ioDev);
        if (!tiles.empty())
            transform_kernel<<<static_cast<unsigned>(tiles.size()), 256, 0, s>>>(
                m_f, m_st.view(), m_seed, m_purpose, dtiles, static_cast<std::uint32_t>(tiles.size()),
                m_ioDev + 4u * m_tileCap, r, C, gf::FastDiv(C), m_st.slotCount(), m_status.dev(), done);
        else
            m_done.completeOnHost();
        cuda::check(cudaGetLastError(), "transform launch");
        ++m_launches;
        return r;
    }
    bool pollsCompletion() const override { return true; }
    bool completed() const override { return m_done.done(); }
    bool advance(cudaStream_t, const Batch&, std::uint32_t& allocated) override
    {
        allocated = 0u;
        const std::uint32_t st = m_done.status();
        if (st != 0u) {
            abort();
            detail::checkStatusWord(st, "transform");
        }
        return false;
    }
    void finish(const Batch&, std::vector<ChunkDescriptor>& outputs) override
    {
        outputs.insert(outputs.end(), m_pending.begin(), m_pending.end());
        m_pending.clear();
    }
    void abort() override
    {
        for (const auto& d : m_pending)
            m_st.ledger().release(d.handle);
        m_pending.clear();
    }

private:
    TStorage& m_st;
    TFunctor m_f;
    std::uint64_t m_seed;
    std::uint32_t m_purpose, m_tile, m_tileCap;
    cuda::HostBuffer<std::uint32_t> m_io;
    std::uint32_t* m_ioDev = nullptr;
    detail::StatusWord m_status;
    detail::CompletionRecord m_done;
    std::vector<ChunkDescriptor> m_pending;
};

template <typename TStorage, typename TFunctor>
class SinkStage final : public Stage {
public:
    SinkStage(TStorage& st, const Config& c, TFunctor f, std::uint32_t purpose)
        : m_st(st), m_f(std::move(f)), m_seed(gf::mix64(c.seed)), m_purpose(purpose),
          m_tiles(static_cast<std::size_t>(c.sinkBatchChunks) * ((c.chunkCapacity + 1023u) / 1024u))
    {
        m_tilesDev = cuda::mappedDevicePointer(m_tiles.data());
    }
    std::uint32_t launch(cudaStream_t s, const Batch& b) override
    {
        const auto tiles = detail::moveTiles(b, 1024u);
        if (tiles.size() > m_tiles.size())
            throw BatchError("sink: tile capacity exceeded");
        std::copy(tiles.begin(), tiles.end(), m_tiles.data());
        const Completion done = m_done.arm();
        if (!tiles.empty())
            sink_kernel<<<static_cast<unsigned>(tiles.size()), 256, 0, s>>>(
                m_f, m_st.view(), m_seed, m_purpose, m_tilesDev, static_cast<std::uint32_t>(tiles.size()),
                m_st.chunkCapacity(), m_st.slotCount(), m_status.dev(), done);
        else
            m_done.completeOnHost();
        cuda::check(cudaGetLastError(), "sink launch");
        ++m_launches;
        return 0u;
    }
    bool pollsCompletion() const override { return true; }
    bool completed() const override { return m_done.done(); }
    bool advance(cudaStream_t, const Batch&, std::uint32_t& allocated) override
    {
        allocated = 0u;
        detail::checkStatusWord(m_done.status(), "sink");
        return false;
    }
    void finish(const Batch&, std::vector<ChunkDescriptor>&) override {}
    void abort() override {}

private:
    TStorage& m_st;
    TFunctor m_f;
    std::uint64_t m_seed;
    std::uint32_t m_purpose;
    cuda::HostBuffer<MoveTile> m_tiles; // mapped: the kernel reads the batch's tiles in place
    MoveTile* m_tilesDev = nullptr;
    detail::StatusWord m_status;
    detail::CompletionRecord m_done;
};

// Dense partition stage. Plain form: classify -> (host) plan -> scatter -> finalise, two device
// stages per batch (Execution.hpp:2363-2725). Fused form: one fused classify->scan->scatter launch
// plus the device finish, output chunks taken from an outputChunkBound reservation at launch.
template <typename TStorage, typename TClassifier, typename TUpdate, typename TBin>
class PartitionStage final : public Stage {
    using View = typename TStorage::View;
    using P = typename TStorage::Payload;
    using Acc = ViewAccess<View>;
    using Cls = ClassifyAdapter<TClassifier, P>;
    using Upd = UpdateAdapter<TUpdate, TBin, P>;
    using Shape = gf::TileShape<256, 4, 2>; // 1024-particle tiles

public:
    PartitionStage(TStorage& st, const Config& c, TClassifier cls, TUpdate upd, std::uint32_t bins,
                   std::uint32_t purpose)
        : m_st(st), m_cls(std::move(cls)), m_upd(std::move(upd)), m_seed(gf::mix64(c.seed)), m_purpose(purpose),
          m_bins(bins), m_C(c.chunkCapacity), m_Q(c.batchChunks), m_fused(c.fused),
          m_direct(c.scatterMode == ScatterMode::Direct),
          m_tileCap(static_cast<std::uint32_t>(c.batchChunks) * ((c.chunkCapacity + kTile - 1u) / kTile)),
          m_bound(checkedOutputChunkBound(static_cast<std::uint64_t>(c.chunkCapacity) * c.batchChunks,
                                          c.chunkCapacity, bins)),
          m_tiles(m_tileCap), m_counts(bins + 1u), m_next(bins), m_table(bins + m_bound), m_status(1),
          m_numOut(1), m_descs(m_bound ? m_bound : 1)
    {
        const std::size_t smemFused = sizeof(P) * Shape::kTile + 4u * Shape::kTile + 4u * Shape::kWarps * bins +
                                      4u * bins * 6u + 4u * (2u * Shape::kThreads + Shape::kWarps + 8u);
        const std::size_t smemScatter = sizeof(P) * Shape::kTile + 4u * Shape::kTile +
                                        4u * Shape::kWarps * bins + 4u * bins * 3u + 4u * (Shape::kWarps + 8u);
        int dev = 0, smemLimit = 0;
        cuda::check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda::check(cudaDeviceGetAttribute(&smemLimit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev),
                    "shared memory limit");
        const auto limit = static_cast<std::size_t>(smemLimit);
        // the hash bin path (per-tile open-addressing tables, Execution.hpp:1208-1502): asked for,
        // more ports than 16-bit dense bins hold, or (automatic path) more than the dense kernels'
        // per-port tables fit in one block
        m_hash = c.binPath == BinPath::hash || bins > Config::denseBinLimit ||
                 (c.binPath == BinPath::automatic && smemFused > limit && smemScatter > limit && !m_direct);
        if (m_hash) {
            if (m_direct)
                throw std::invalid_argument("graphflow::PartitionStage: the hash path has no direct scatter");
            m_fused = false;
        } else {
            // many ports: the fused kernel's per-port tables no longer fit one block; the plain form's do
            if (m_fused && smemFused > limit)
                m_fused = false;
            if (!m_fused && !m_direct && smemScatter > limit)
                throw std::invalid_argument("graphflow::PartitionStage: " + std::to_string(bins) +
                                            " ports need more shared memory per block than the device has");
        }
        if (m_fused) {
            m_maxK = m_Q;
            m_portChunks = cuda::Buffer<unsigned long long>(static_cast<std::size_t>(bins) * m_maxK);
            cuda::check(cudaMemset(m_portChunks.data(), 0, m_portChunks.size() * 8), "memset");
            gf_fused_scratch_bytes(m_tileCap, bins, &m_scratchBytes);
            // one mirrored buffer per stage (u32 words): [numOut | totals | descs | tiles | reserved |
            // status | pad | fused scratch (control block, descriptors)]. A batch uploads tiles through
            // the control block's three reset words (zeroing status and those words; the persistent
            // epoch after them is not touched) and downloads numOut through status: one copy each way.
            m_oTotals = 1u;
            m_oDescs = m_oTotals + bins;
            m_oTiles = m_oDescs + 3u * (m_bound ? m_bound : 1u);
            m_oReserved = m_oTiles + 3u * m_tileCap;
            m_oStatus = m_oReserved + (m_bound ? m_bound : 1u);
            m_oCtl = (m_oStatus + 1u + 15u) & ~15u; // 64-byte aligned control block
            static_assert(sizeof(gf_tile) == 12 && sizeof(gf_out_desc) == 12, "packed layout");
            static_assert(gf::kFusedCtlResetBytes == 12, "three reset words");
            m_io = detail::Staged<std::uint32_t>(m_oCtl + (m_scratchBytes + 3u) / 4u);
            cuda::check(cudaMemset(m_io.dev.data(), 0, m_io.dev.size() * 4u), "memset");
            std::fill(m_io.host.data(), m_io.host.data() + m_io.host.size(), 0u);
            // per batch, no copies and no event: the kernel reads its tiles and reserved chunks from
            // mapped pinned memory and its finishing CTA writes a completion record there (status,
            // output count, totals, descriptors, then the batch's sequence number), which the runner
            // polls with a plain load; the launch counters reset themselves
            m_hin = cuda::HostBuffer<std::uint32_t>(3u * m_tileCap + (m_bound ? m_bound : 1u));
            m_rec = cuda::HostBuffer<std::uint32_t>(3u + bins + 3u * (m_bound ? m_bound : 1u));
            std::fill(m_rec.data(), m_rec.data() + m_rec.size(), 0u);
            m_hinDev = cuda::mappedDevicePointer(m_hin.data());
            m_recDev = cuda::mappedDevicePointer(m_rec.data());
        } else {
            m_binIds = cuda::Buffer<std::uint32_t>(st.slotCount());
        }
        m_smemFused = smemFused;
        m_smemScatter = smemScatter;
        if (m_fused)
            cuda::check(cudaFuncSetAttribute(gf::fused_partition_kernel<Shape, Acc, Cls, Upd>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smemFused)),
                        "partition stage: fused kernel attribute");
        if (!m_hash && !m_direct && smemScatter <= limit)
            cuda::check(cudaFuncSetAttribute(gf::scatter_kernel<Shape, Acc, Upd>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smemScatter)),
                        "partition stage: scatter kernel attribute");
        if (m_hash) {
            constexpr std::size_t E = 2u * Shape::kTile; // table entries per tile
            m_smemScatter = sizeof(P) * Shape::kTile + 4u * Shape::kTile + 4u * 4u * E + 4u * (Shape::kWarps + 2u) + 16u;
            cuda::check(cudaFuncSetAttribute(gf::hash_scatter_kernel<Shape, Acc, Upd, Cls>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(m_smemScatter)),
                        "partition stage: hash scatter kernel attribute");
        }
    }

    std::uint32_t launch(cudaStream_t s, const Batch& b) override
    {
        if (m_failed)
            throw std::logic_error("graphflow::PartitionStage: single-use after a failed batch");
        if (b.chunks.empty() || b.chunks.size() > m_Q)
            throw BatchError("partition: batch must hold 1..batchChunks chunks");
        m_stage = 0;
        m_pending.clear();
        m_n = b.particles();
        m_numTiles = 0;
        for (const auto& c : b.chunks)
            for (std::uint32_t off = 0; off < c.fill; off += kTile) {
                if (m_numTiles >= m_tileCap)
                    throw BatchError("partition: tile descriptor capacity exceeded");
                m_tiles.host[m_numTiles++] = gf_tile{c.handle.index, off, c.fill - off < kTile ? c.fill - off : kTile};
            }
        const Acc acc{m_st.view()};
        ++m_launches;
        if (m_fused) {
            std::uint32_t* io = m_io.dev.data();
            std::uint32_t* status = io + m_oStatus;
            const Cls cls{m_cls, m_seed, m_purpose, status};
            const Upd upd{m_upd, m_purpose + 1u, status};
            const std::uint32_t bound = checkedOutputChunkBound(m_n, m_C, m_bins);
            std::memcpy(m_hin.data(), m_tiles.host.data(), sizeof(gf_tile) * m_numTiles);
            m_reserved.clear();
            for (std::uint32_t k = 0; k < bound; ++k) {
                m_reserved.push_back(m_st.ledger().acquire());
                m_hin.data()[3u * m_tileCap + k] = m_reserved.back().index;
            }
            ++m_seq;
            auto* ctl = reinterpret_cast<gf::FusedCtl*>(io + m_oCtl);
            auto* desc = reinterpret_cast<unsigned long long*>(ctl + 1);
            auto* tiles = reinterpret_cast<const gf_tile*>(m_hinDev);
            auto* descs = reinterpret_cast<gf_out_desc*>(io + m_oDescs);
            if (m_numTiles) {
                // the launch's last CTA builds the table and descriptors and publishes the record
                gf::InlineFinish fin{m_table.dev.data(), descs, m_bound, io};
                fin.done_rec = m_recDev;
                fin.done_seq = m_seq;
                gf::fused_partition_kernel<Shape, Acc, Cls, Upd><<<m_numTiles, Shape::kThreads, m_smemFused, s>>>(
                    acc, cls, upd, m_seed, m_C, gf::FastDiv(m_C), m_st.slotCount(), tiles, m_numTiles, m_bins,
                    m_hinDev + 3u * m_tileCap, bound, io + m_oTotals, m_portChunks.data(), m_maxK, ctl, desc, status,
                    fin, gf::NoPost{});
                cuda::check(cudaGetLastError(), "fused partition kernel launch");
            } else {
                // an empty batch: nothing to run, the record is complete at once
                std::uint32_t* rec = m_rec.data();
                std::fill(rec + 1, rec + 3 + m_bins, 0u);
                reinterpret_cast<volatile std::uint32_t*>(rec)[0] = m_seq;
            }
            return bound;
        }
        m_tiles.upload(s, m_numTiles);
        cuda::check(cudaMemsetAsync(m_status.dev.data(), 0, 4, s), "memset");
        const Cls cls{m_cls, m_seed, m_purpose, m_status.dev.data()};
        cuda::check(cudaMemsetAsync(m_counts.dev.data(), 0, 4u * (m_bins + 1u), s), "memset");
        if (m_numTiles && m_hash)
            gf::hash_classify_kernel<Shape, Acc, Cls><<<m_numTiles, Shape::kThreads, 0, s>>>(
                acc, cls, m_C, m_st.slotCount(), m_tiles.dev.data(), m_numTiles, m_bins, m_binIds.data(),
                m_counts.dev.data(), m_status.dev.data());
        else if (m_numTiles)
            gf::classify_kernel<Shape, Acc, Cls><<<m_numTiles, Shape::kThreads, 4u * m_bins, s>>>(
                acc, cls, m_C, m_st.slotCount(), m_tiles.dev.data(), m_numTiles, m_bins, m_binIds.data(),
                m_counts.dev.data(), m_status.dev.data());
        cuda::check(cudaGetLastError(), "classify launch");
        m_status.download(s, 1);
        m_counts.download(s, m_bins + 1u);
        return 0u;
    }

    bool pollsCompletion() const override { return m_fused; }
    bool completed() const override
    {
        const bool done = reinterpret_cast<const volatile std::uint32_t*>(m_rec.data())[0] == m_seq;
        if (done)
            std::atomic_thread_fence(std::memory_order_acquire);
        return done;
    }

    bool advance(cudaStream_t s, const Batch& b, std::uint32_t& allocated) override
    {
        allocated = 0u;
        try {
            if (m_fused)
                return finishFused(b);
            if (m_stage == 0) {
                planAndScatter(s, b, allocated);
                m_stage = 1;
                return true;
            }
            finalise();
            m_stage = 0;
            return false;
        } catch (...) {
            abort();
            throw;
        }
    }

    void finish(const Batch&, std::vector<ChunkDescriptor>& outputs) override
    {
        outputs.insert(outputs.end(), m_pending.begin(), m_pending.end());
        m_pending.clear();
    }

    void abort() override
    {
        for (const auto& d : m_pending)
            if (m_st.ledger().valid(d.handle))
                m_st.ledger().release(d.handle);
        m_pending.clear();
        for (const auto& h : m_reserved)
            if (m_st.ledger().valid(h))
                m_st.ledger().release(h);
        m_reserved.clear();
        m_failed = true;
    }

private:
    static constexpr std::uint32_t kTile = Shape::kTile;

    bool finishFused(const Batch&)
    {
        const std::uint32_t* rec = m_rec.data();
        detail::checkStatusWord(rec[1], "fused partition");
        const std::uint32_t r = rec[2];
        std::uint64_t total = 0;
        for (std::uint32_t b = 0; b < m_bins; ++b)
            total += rec[3u + b];
        if (total != m_n)
            throw BatchError("fused partition: classified particle count does not match the batch");
        // reservation slot of every reserved chunk index (a flat table over the pool, cleared after use)
        if (m_slotOf.size() != m_st.ledger().numChunks())
            m_slotOf.assign(m_st.ledger().numChunks(), -1);
        for (std::size_t k = 0; k < m_reserved.size(); ++k)
            m_slotOf[m_reserved[k].index] = static_cast<std::int32_t>(k);
        struct Clear { // on every exit: the table is all -1 again
            std::vector<std::int32_t>& t;
            const std::vector<ChunkHandle>& r;
            ~Clear()
            {
                for (const auto& h : r)
                    t[h.index] = -1;
            }
        } clear{m_slotOf, m_reservedCopy};
        m_reservedCopy = m_reserved;
        if (r > m_bound)
            throw BatchError("fused partition: more output chunks than the reservation bound");
        const gf_out_desc* d = reinterpret_cast<const gf_out_desc*>(rec + 3u + m_bins);
        std::vector<bool>& used = m_usedSlot;
        used.assign(m_reserved.size(), false);
        for (std::uint32_t i = 0; i < r; ++i) {
            const std::int32_t k = d[i].chunk_index < m_slotOf.size() ? m_slotOf[d[i].chunk_index] : -1;
            if (k < 0 || used[static_cast<std::size_t>(k)])
                throw BatchError("fused partition: output chunk outside the reservation");
            used[static_cast<std::size_t>(k)] = true;
            m_pending.push_back(ChunkDescriptor{m_reserved[static_cast<std::size_t>(k)], d[i].fill, d[i].bin});
        }
        for (std::size_t k = 0; k < m_reserved.size(); ++k)
            if (!used[k])
                m_st.ledger().release(m_reserved[k]);
        m_reserved.clear();
        return false;
    }

    void planAndScatter(cudaStream_t s, const Batch& b, std::uint32_t& allocated)
    {
        detail::checkStatusWord(m_status.host[0], "partition classify");
        if (m_counts.host[m_bins] != 0u)
            throw BatchError("partition classify: device status reports an invalid classifier result");
        std::uint64_t total = 0;
        for (std::uint32_t k = 0; k < m_bins; ++k)
            total += m_counts.host[k];
        if (total != b.particles())
            throw BatchError("partition classify: classified particle count does not match the batch");
        std::vector<std::uint32_t> base(m_bins), fills(m_bound ? m_bound : 1);
        std::uint32_t r = 0;
        throw_on(gf_plan_dense(m_counts.host.data(), m_bins, m_C, base.data(), fills.data(),
                               static_cast<std::uint32_t>(fills.size()), &r),
                 "planDenseBins");
        if (r > m_bound)
            throw BatchError("partition plan: exact chunk count exceeds the reservation bound");
        for (std::uint32_t k = 0; k < m_bins; ++k)
            m_table.host[k] = base[k];
        std::uint32_t f = 0;
        for (std::uint32_t bin = 0; bin < m_bins; ++bin) {
            const std::uint32_t chunks = (m_counts.host[bin] + m_C - 1u) / m_C;
            for (std::uint32_t k = 0; k < chunks; ++k, ++f) {
                const ChunkHandle h = m_st.ledger().acquire();
                m_table.host[m_bins + f] = h.index;
                m_pending.push_back(ChunkDescriptor{h, fills[f], bin});
            }
        }
        allocated = r;
        m_totals0.assign(m_counts.host.data(), m_counts.host.data() + m_bins);
        m_table.upload(s, m_bins + r);
        cuda::check(cudaMemsetAsync(m_next.dev.data(), 0, 4u * m_bins, s), "memset");
        cuda::check(cudaMemsetAsync(m_status.dev.data(), 0, 4, s), "memset");
        if (m_numTiles) {
            const Acc acc{m_st.view()};
            const Upd upd{m_upd, m_purpose + 1u, m_status.dev.data()};
            if (m_hash) // per-tile tables again, one range per occupied entry (Execution.hpp:1336-1502)
                gf::hash_scatter_kernel<Shape, Acc, Upd, Cls><<<m_numTiles, Shape::kThreads, m_smemScatter, s>>>(
                    acc, Cls{m_cls, m_seed, m_purpose, m_status.dev.data()}, upd, m_seed, m_C, gf::FastDiv(m_C),
                    m_st.slotCount(), m_tiles.dev.data(), m_numTiles, m_bins, m_binIds.data(), m_table.dev.data(),
                    m_next.dev.data(), m_counts.dev.data(), m_status.dev.data());
            else if (m_direct) // one device atomic per particle (Execution.hpp:1034-1095)
                gf::scatter_direct_kernel<Shape, Acc, Upd><<<m_numTiles, Shape::kThreads, 0, s>>>(
                    acc, upd, m_seed, m_C, gf::FastDiv(m_C), m_st.slotCount(), m_tiles.dev.data(), m_numTiles,
                    m_bins, m_binIds.data(), m_table.dev.data(), m_next.dev.data(), m_counts.dev.data(),
                    m_status.dev.data());
            else
                gf::scatter_kernel<Shape, Acc, Upd><<<m_numTiles, Shape::kThreads, m_smemScatter, s>>>(
                    acc, upd, m_seed, m_C, gf::FastDiv(m_C), m_st.slotCount(), m_tiles.dev.data(), m_numTiles,
                    m_bins, m_binIds.data(), m_table.dev.data(), m_next.dev.data(), m_counts.dev.data(),
                    m_status.dev.data());
            cuda::check(cudaGetLastError(), "scatter launch");
            ++m_launches;
        }
        m_status.download(s, 1);
        m_counts.download(s, m_bins + 1u);
        m_next.download(s, m_bins);
    }

    void finalise()
    {
        detail::checkStatusWord(m_status.host[0], "partition scatter");
        if (m_counts.host[m_bins] != 0u)
            throw BatchError("partition scatter: device status reports a checked updater overflow");
        for (std::uint32_t k = 0; k < m_bins; ++k)
            if (m_next.host[k] != m_totals0[k])
                throw BatchError("partition scatter: next[bin] does not match total[bin]");
    }

    TStorage& m_st;
    TClassifier m_cls;
    TUpdate m_upd;
    std::uint64_t m_seed;
    std::uint32_t m_purpose, m_bins, m_C, m_Q;
    bool m_fused;
    bool m_direct;       // plain form: ScatterMode::Direct
    bool m_hash = false; // plain form through the per-tile hash tables
    std::uint32_t m_tileCap, m_bound;
    detail::Staged<gf_tile> m_tiles;
    detail::Staged<std::uint32_t> m_counts, m_next, m_table, m_status, m_numOut;
    detail::Staged<gf_out_desc> m_descs;
    detail::Staged<std::uint32_t> m_io; // fused form: the packed per-batch buffer (layout in the constructor)
    cuda::HostBuffer<std::uint32_t> m_hin, m_rec; // fused form: mapped tiles + reserved chunks, completion record
    std::uint32_t* m_hinDev = nullptr;
    std::uint32_t* m_recDev = nullptr;
    std::uint32_t m_seq = 0;
    std::uint32_t m_oTotals = 0, m_oDescs = 0, m_oTiles = 0, m_oReserved = 0, m_oStatus = 0, m_oCtl = 0;
    cuda::Buffer<std::uint32_t> m_binIds;
    cuda::Buffer<unsigned long long> m_portChunks;
    std::uint64_t m_scratchBytes = 0;
    std::uint32_t m_maxK = 1;
    std::size_t m_smemFused = 0, m_smemScatter = 0;
    std::uint32_t m_stage = 0, m_numTiles = 0;
    std::uint64_t m_n = 0;
    std::vector<ChunkDescriptor> m_pending;
    std::vector<ChunkHandle> m_reserved, m_reservedCopy;
    std::vector<std::int32_t> m_slotOf; // fused form: reservation slot by chunk index, -1 elsewhere
    std::vector<bool> m_usedSlot;
    std::vector<std::uint32_t> m_totals0;
    bool m_failed = false;
};

// Several fused partition nodes of one classifier and updater type, run as one runner node.
// Each input chunk carries its member node in ChunkDescriptor::bin (the runner's route tags). A
// launch cuts every member's chunks, in arrival order, into batches of at most Q chunks, reserves
// outputChunkBound output chunks per batch and runs all of them in one multi-batch fused kernel
// (gf::fused_partition_multi_kernel): the per-node batches of GraphRunner.hpp:985-1133 drained by a
// single launch. Every batch's plan, table and outputs are those its node would produce alone;
// outputs carry bin = member * B + port for the group's route table.
template <typename TStorage, typename TClassifier, typename TUpdate, typename TBin>
class PartitionGroupStage final : public Stage {
    using View = typename TStorage::View;
    using P = typename TStorage::Payload;
    using Acc = ViewAccess<View>;
    using Cls = ClassifyAdapter<TClassifier, P>;
    using Upd = UpdateAdapter<TUpdate, TBin, P>;
    using Shape = gf::TileShape<256, 4, 2>; // 1024-particle tiles
    static constexpr std::uint32_t kTile = 1024u;

public:
    static std::size_t smemBytes(std::uint32_t bins)
    {
        return sizeof(P) * Shape::kTile + 4u * Shape::kTile + 4u * Shape::kWarps * bins + 4u * bins * 6u +
               4u * (2u * Shape::kThreads + Shape::kWarps + 8u);
    }
    // The group runs the dense fused kernel only: fused form, shared-memory staging, dense bins
    // whose per-port tables fit one block.
    static bool feasible(const Config& c, std::uint32_t bins)
    {
        if (!c.fused || c.scatterMode == ScatterMode::Direct || c.binPath == BinPath::hash ||
            bins > Config::denseBinLimit)
            return false;
        int dev = 0, limit = 0;
        cuda::check(cudaGetDevice(&dev), "cudaGetDevice");
        cuda::check(cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "smem limit");
        return smemBytes(bins) <= static_cast<std::size_t>(limit);
    }

    PartitionGroupStage(TStorage& st, const Config& c, std::uint32_t bins)
        : m_st(st), m_seed(gf::mix64(c.seed)), m_bins(bins), m_C(c.chunkCapacity), m_Q(c.batchChunks),
          m_maxChunks(c.groupChunks), m_maxBatches(maxBatchesFor(c, bins)),
          m_tilesPerChunk((c.chunkCapacity + kTile - 1u) / kTile),
          m_maxTiles(c.groupChunks * ((c.chunkCapacity + kTile - 1u) / kTile)),
          m_tilesPerBatch(c.batchChunks * ((c.chunkCapacity + kTile - 1u) / kTile)),
          m_boundMax(checkedOutputChunkBound(static_cast<std::uint64_t>(c.chunkCapacity) * c.batchChunks,
                                             c.chunkCapacity, bins))
    {
        static_assert(sizeof(gf::MultiBatch) % 8u == 0u, "8-byte aligned batch records");
        static_assert(sizeof(gf_tile) == 12 && sizeof(gf_out_desc) == 12, "packed layout");
        if (!feasible(c, bins))
            throw std::invalid_argument("graphflow::PartitionGroupStage: the fused dense kernel does not apply");
        m_portChunks = cuda::Buffer<unsigned long long>(static_cast<std::size_t>(m_maxBatches) * bins * m_Q);
        m_desc = cuda::Buffer<unsigned long long>(static_cast<std::size_t>(m_maxBatches) * m_tilesPerBatch * bins);
        m_totals = cuda::Buffer<std::uint32_t>(static_cast<std::size_t>(m_maxBatches) * bins);
        m_table = cuda::Buffer<std::uint32_t>(static_cast<std::size_t>(m_maxBatches) * (bins + m_boundMax));
        cuda::check(cudaMemset(m_portChunks.data(), 0, m_portChunks.size() * 8u), "memset");
        cuda::check(cudaMemset(m_desc.data(), 0, m_desc.size() * 8u), "memset");
        // a launch makes no copy and records no event: the kernel reads its payload (tiles, tile
        // batch, batch records, reserved chunks) from mapped pinned memory, every batch's finish
        // writes its output count and descriptors into the mapped record [sequence | status |
        // numOut[maxBatches] | descs[maxBatches][boundMax]], and the last batch to finish writes
        // the status and then the sequence number, which the runner polls. The device words
        // [status | pad | control block (4) | per-batch counters (2 each)] reset themselves.
        m_dev = cuda::Buffer<std::uint32_t>(8u + 2u * static_cast<std::size_t>(m_maxBatches));
        cuda::check(cudaMemset(m_dev.data(), 0, m_dev.size() * 4u), "memset");
        m_oNum = 2u;
        m_oDescs = m_oNum + m_maxBatches;
        m_rec = cuda::HostBuffer<std::uint32_t>(m_oDescs + 3u * static_cast<std::size_t>(m_maxBatches) * m_boundMax);
        std::fill(m_rec.data(), m_rec.data() + m_rec.size(), 0u);
        const std::size_t payMax = 4u * static_cast<std::size_t>(m_maxTiles) +
                                   m_maxBatches * (sizeof(gf::MultiBatch) / 4u + m_boundMax) + 4u;
        m_pay = cuda::HostBuffer<std::uint32_t>(payMax);
        m_payDev = cuda::mappedDevicePointer(m_pay.data());
        m_recDev = cuda::mappedDevicePointer(m_rec.data());
        m_smem = smemBytes(bins);
        cuda::check(cudaFuncSetAttribute(gf::fused_partition_multi_kernel<Shape, Acc, Cls, Upd>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(m_smem)),
                    "partition group: kernel attribute");
    }

    // Batches one launch holds: one per input chunk at most, and the batches' look-back descriptor
    // scratch (tiles x ports x 8 bytes each) within 64 MiB.
    static std::uint32_t maxBatchesFor(const Config& c, std::uint32_t bins)
    {
        const std::uint64_t perBatch = static_cast<std::uint64_t>(c.batchChunks) *
                                       ((c.chunkCapacity + kTile - 1u) / kTile) * bins * 8u;
        const std::uint64_t cap = std::max<std::uint64_t>(1u, (64ull << 20) / std::max<std::uint64_t>(perBatch, 1u));
        return static_cast<std::uint32_t>(std::min<std::uint64_t>(c.groupChunks, cap));
    }

    // A member node's classifier, updater and stream purpose; its index is the route tag of the
    // chunks routed to it.
    std::uint32_t addMember(TClassifier cls, TUpdate upd, std::uint32_t purpose)
    {
        std::uint32_t* status = m_dev.data();
        m_cls.push_back(Cls{cls, m_seed, purpose, status});
        m_upd.push_back(Upd{upd, purpose + 1u, status});
        m_membersDirty = true;
        return static_cast<std::uint32_t>(m_cls.size() - 1u);
    }
    std::uint32_t members() const { return static_cast<std::uint32_t>(m_cls.size()); }

    bool plansBatches() const override { return true; }
    bool pollsCompletion() const override { return true; }
    bool completed() const override
    {
        const bool done = reinterpret_cast<const volatile std::uint32_t*>(m_rec.data())[0] == m_seq;
        if (done)
            std::atomic_thread_fence(std::memory_order_acquire);
        return done;
    }
    std::uint32_t lastLaunchBatches() const override { return static_cast<std::uint32_t>(m_sub.size()); }

    // The longest prefix of `ready` (at most groupChunks chunks, tiles and batches within the
    // launch's capacity) whose batches' output bounds fit `available`.
    std::size_t planBatch(const std::deque<ChunkDescriptor>& ready, std::uint32_t available,
                          std::uint32_t& reserve) const override
    {
        reserve = 0u;
        const std::size_t m = m_cls.size();
        m_openChunks.assign(m, 0u);
        m_openN.assign(m, 0u);
        std::uint64_t closed = 0, open = 0;
        std::uint32_t batches = 0, tiles = 0;
        std::size_t take = 0;
        const std::size_t limit = std::min<std::size_t>(ready.size(), m_maxChunks);
        for (std::size_t j = 0; j < limit; ++j) {
            const ChunkDescriptor& d = ready[j];
            if (d.bin >= m)
                break; // not a member's chunk: launch() rejects it
            const std::uint32_t mb = d.bin;
            const std::uint32_t t = (d.fill + kTile - 1u) / kTile;
            std::uint64_t o = open, c = closed;
            std::uint32_t nb = batches;
            if (m_openChunks[mb] == 0u || m_openChunks[mb] == m_Q) {
                if (m_openChunks[mb] == m_Q) {
                    const std::uint32_t bnd = checkedOutputChunkBound(m_openN[mb], m_C, m_bins);
                    o -= bnd;
                    c += bnd;
                }
                ++nb;
            } else {
                o -= checkedOutputChunkBound(m_openN[mb], m_C, m_bins);
            }
            const std::uint64_t n = (m_openChunks[mb] == m_Q ? 0u : m_openN[mb]) + d.fill;
            o += checkedOutputChunkBound(n, m_C, m_bins);
            if (c + o > available || nb > m_maxBatches || tiles + t > m_maxTiles)
                break;
            open = o;
            closed = c;
            batches = nb;
            tiles += t;
            m_openChunks[mb] = m_openChunks[mb] == m_Q ? 1u : m_openChunks[mb] + 1u;
            m_openN[mb] = n;
            take = j + 1u;
        }
        reserve = static_cast<std::uint32_t>(closed + open);
        return take;
    }

    std::uint32_t launch(cudaStream_t s, const Batch& b) override
    {
        if (m_failed)
            throw std::logic_error("graphflow::PartitionGroupStage: single-use after a failed batch");
        if (m_cls.empty())
            throw std::logic_error("graphflow::PartitionGroupStage: no member nodes");
        ++m_launches;
        if (m_membersDirty) {
            m_clsDev = cuda::Buffer<Cls>(m_cls.size());
            m_updDev = cuda::Buffer<Upd>(m_upd.size());
            cuda::check(cudaMemcpy(m_clsDev.data(), m_cls.data(), sizeof(Cls) * m_cls.size(), cudaMemcpyHostToDevice),
                        "H2D");
            cuda::check(cudaMemcpy(m_updDev.data(), m_upd.data(), sizeof(Upd) * m_upd.size(), cudaMemcpyHostToDevice),
                        "H2D");
            m_membersDirty = false;
        }
        // batches: every member's chunks in arrival order, at most Q per batch
        m_sub.clear();
        m_cur.assign(m_cls.size(), -1);
        for (const auto& c : b.chunks) {
            if (c.bin >= m_cls.size())
                throw BatchError("partition group: chunk routed to an unknown member");
            int& k = m_cur[c.bin];
            if (k < 0 || m_sub[static_cast<std::size_t>(k)].chunks.size() == m_Q) {
                k = static_cast<int>(m_sub.size());
                m_sub.push_back(Sub{c.bin, {}, 0u, 0u, 0u, 0u, 0u});
            }
            m_sub[static_cast<std::size_t>(k)].chunks.push_back(c);
        }
        if (m_sub.size() > m_maxBatches)
            throw BatchError("partition group: more batches than one launch holds");
        // reservations, tiles and batch records
        std::uint32_t* h = m_pay.data();
        std::uint32_t* d = m_payDev;
        std::uint32_t nTiles = 0, nReserved = 0, live = 0;
        m_reserved.clear();
        for (auto& sb : m_sub) {
            sb.n = 0u;
            for (const auto& c : sb.chunks)
                sb.n += c.fill;
            sb.bound = checkedOutputChunkBound(sb.n, m_C, m_bins);
            sb.resBegin = nReserved;
            for (std::uint32_t k = 0; k < sb.bound; ++k)
                m_reserved.push_back(m_st.ledger().acquire());
            nReserved += sb.bound;
            sb.tileBegin = nTiles;
            for (const auto& c : sb.chunks)
                nTiles += (c.fill + kTile - 1u) / kTile;
            sb.tiles = nTiles - sb.tileBegin;
            live += sb.tiles != 0u ? 1u : 0u;
        }
        if (nTiles > m_maxTiles)
            throw BatchError("partition group: more tiles than one launch holds");
        const std::uint32_t nb = static_cast<std::uint32_t>(m_sub.size());
        const std::uint32_t oTiles = 0u, oTileBatch = oTiles + 3u * nTiles;
        const std::uint32_t oBatches = (oTileBatch + nTiles + 1u) & ~1u;
        const std::uint32_t oRes = oBatches + nb * static_cast<std::uint32_t>(sizeof(gf::MultiBatch) / 4u);
        auto* tiles = reinterpret_cast<gf_tile*>(h + oTiles);
        auto* recs = reinterpret_cast<gf::MultiBatch*>(h + oBatches);
        std::uint32_t* rec = m_rec.data();
        std::uint32_t t = 0;
        for (std::uint32_t i = 0; i < nb; ++i) {
            const Sub& sb = m_sub[i];
            for (const auto& c : sb.chunks)
                for (std::uint32_t off = 0; off < c.fill; off += kTile) {
                    tiles[t] = gf_tile{c.handle.index, off, c.fill - off < kTile ? c.fill - off : kTile};
                    h[oTileBatch + t] = i;
                    ++t;
                }
            for (std::uint32_t k = 0; k < sb.bound; ++k)
                h[oRes + sb.resBegin + k] = m_reserved[sb.resBegin + k].index;
            gf::MultiBatch r{};
            r.tile_begin = sb.tileBegin;
            r.n_tiles = sb.tiles;
            r.member = sb.member;
            r.n_reserved = sb.bound;
            r.reserved = d + oRes + sb.resBegin;
            r.totals = m_totals.data() + static_cast<std::size_t>(i) * m_bins;
            r.port_chunks = m_portChunks.data() + static_cast<std::size_t>(i) * m_bins * m_Q;
            r.desc = m_desc.data() + static_cast<std::size_t>(i) * m_tilesPerBatch * m_bins;
            r.counters = m_dev.data() + 8u + 2u * i;
            r.table = m_table.data() + static_cast<std::size_t>(i) * (m_bins + m_boundMax);
            r.descs = reinterpret_cast<gf_out_desc*>(m_recDev + m_oDescs) + static_cast<std::size_t>(i) * m_boundMax;
            r.desc_cap = m_boundMax;
            r.num_out = m_recDev + m_oNum + i;
            recs[i] = r;
            rec[m_oNum + i] = 0u;
        }
        ++m_seq;
        if (live != 0u) {
            const Acc acc{m_st.view()};
            gf::fused_partition_multi_kernel<Shape, Acc, Cls, Upd><<<nTiles, Shape::kThreads, m_smem, s>>>(
                acc, m_clsDev.data(), m_updDev.data(), m_seed, m_C, gf::FastDiv(m_C), m_st.slotCount(),
                reinterpret_cast<const gf_tile*>(d + oTiles), d + oTileBatch, nTiles, m_bins,
                reinterpret_cast<const gf::MultiBatch*>(d + oBatches), nb, m_Q,
                reinterpret_cast<gf::FusedCtl*>(m_dev.data() + 4u), m_dev.data(), m_recDev, m_seq, live);
            cuda::check(cudaGetLastError(), "partition group launch");
        } else {
            rec[1] = 0u; // no particle: the record is complete at once
            reinterpret_cast<volatile std::uint32_t*>(rec)[0] = m_seq;
        }
        return nReserved;
    }

    bool advance(cudaStream_t, const Batch&, std::uint32_t& allocated) override
    {
        allocated = 0u;
        detail::checkStatusWord(m_rec.data()[1], "partition group");
        return false;
    }

    void finish(const Batch&, std::vector<ChunkDescriptor>& outputs) override
    {
        if (m_slotOf.size() != m_st.ledger().numChunks())
            m_slotOf.assign(m_st.ledger().numChunks(), -1);
        for (std::size_t k = 0; k < m_reserved.size(); ++k)
            m_slotOf[m_reserved[k].index] = static_cast<std::int32_t>(k);
        m_used.assign(m_reserved.size(), false);
        std::vector<ChunkHandle> reserved = std::move(m_reserved);
        m_reserved.clear();
        struct Clear { // on every exit: the table is all -1 again, unused reservations are released
            std::vector<std::int32_t>& slot;
            const std::vector<ChunkHandle>& r;
            const std::vector<bool>& used;
            ChunkLedger& ledger;
            bool committed = false; // outputs handed to the runner; otherwise every reservation goes back
            ~Clear()
            {
                for (std::size_t k = 0; k < r.size(); ++k) {
                    slot[r[k].index] = -1;
                    if ((!committed || !used[k]) && ledger.valid(r[k]))
                        ledger.release(r[k]);
                }
            }
        } clear{m_slotOf, reserved, m_used, m_st.ledger()};
        std::vector<ChunkDescriptor> out;
        const auto* descs = reinterpret_cast<const gf_out_desc*>(m_rec.data() + m_oDescs);
        for (std::size_t i = 0; i < m_sub.size(); ++i) {
            const Sub& sb = m_sub[i];
            if (sb.n == 0u)
                continue;
            const std::uint32_t r = m_rec.data()[m_oNum + i];
            if (r > sb.bound)
                throw BatchError("partition group: more output chunks than the reservation bound");
            std::uint64_t placed = 0;
            const gf_out_desc* d = descs + i * m_boundMax;
            for (std::uint32_t q = 0; q < r; ++q) {
                const std::int32_t k = d[q].chunk_index < m_slotOf.size() ? m_slotOf[d[q].chunk_index] : -1;
                if (k < static_cast<std::int32_t>(sb.resBegin) || k >= static_cast<std::int32_t>(sb.resBegin + sb.bound) ||
                    m_used[static_cast<std::size_t>(k)])
                    throw BatchError("partition group: output chunk outside the batch's reservation");
                if (d[q].bin >= m_bins)
                    throw BatchError("partition group: output bin out of range");
                m_used[static_cast<std::size_t>(k)] = true;
                placed += d[q].fill;
                out.push_back(ChunkDescriptor{reserved[static_cast<std::size_t>(k)], d[q].fill,
                                              sb.member * m_bins + d[q].bin});
            }
            if (placed != sb.n)
                throw BatchError("partition group: placed particle count does not match the batch");
        }
        outputs.insert(outputs.end(), out.begin(), out.end());
        clear.committed = true;
        m_sub.clear();
    }

    void abort() override
    {
        m_failed = true;
        for (const auto& h : m_reserved)
            if (m_st.ledger().valid(h))
                m_st.ledger().release(h);
        m_reserved.clear();
        m_sub.clear();
    }

private:
    struct Sub {
        std::uint32_t member;
        std::vector<ChunkDescriptor> chunks;
        std::uint64_t n;
        std::uint32_t bound, resBegin, tileBegin, tiles;
    };

    TStorage& m_st;
    std::uint64_t m_seed;
    std::uint32_t m_bins, m_C, m_Q, m_maxChunks, m_maxBatches, m_tilesPerChunk, m_maxTiles, m_tilesPerBatch, m_boundMax;
    std::vector<Cls> m_cls;
    std::vector<Upd> m_upd;
    cuda::Buffer<Cls> m_clsDev;
    cuda::Buffer<Upd> m_updDev;
    bool m_membersDirty = true;
    cuda::Buffer<unsigned long long> m_portChunks, m_desc;
    cuda::Buffer<std::uint32_t> m_totals, m_table;
    cuda::Buffer<std::uint32_t> m_dev;
    cuda::HostBuffer<std::uint32_t> m_pay, m_rec;
    std::uint32_t* m_payDev = nullptr;
    std::uint32_t* m_recDev = nullptr;
    std::uint32_t m_oNum = 0, m_oDescs = 0;
    std::size_t m_smem = 0;
    std::uint32_t m_seq = 0;
    std::vector<Sub> m_sub;
    std::vector<int> m_cur;
    std::vector<ChunkHandle> m_reserved;
    std::vector<std::int32_t> m_slotOf;
    std::vector<bool> m_used;
    mutable std::vector<std::uint32_t> m_openChunks;
    mutable std::vector<std::uint64_t> m_openN;
    bool m_failed = false;
};

} // namespace graphflow
