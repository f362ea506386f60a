// Host-side core of the graphflow_b200 C++ front end: errors, tuning and resolved configuration,
// scheduler statistics, chunk handles/descriptors and the chunk pool ledger.
//
// Reference (paths inside graphFlow's include/graphFlow): flow/Tuning.hpp:27-145,
// core/Config.hpp:60-349 (validation subset on the hot path), sched/GraphRunner.hpp:154-252
// (SchedulerStats), core/Chunk.hpp:19-37, core/ChunkPool.hpp / core/ChunkLedger.hpp (free list,
// generations, reader leases).
#pragma once

#include <chrono>
#include <cstdint>
#include <deque>
#include <limits>
#include <optional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "graphflow_b200.h"

namespace graphflow {

// ---- errors (flow/Execution.hpp BatchError, sched/GraphRunner.hpp SchedulerStallError) ----
struct BatchError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct SchedulerStallError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void throw_on(gf_status rc, const char* what)
{
    switch (rc) {
    case GF_OK:
        return;
    case GF_ERR_ARGUMENT:
        throw std::invalid_argument(std::string(what) + ": invalid argument");
    case GF_ERR_RANGE:
        throw std::overflow_error(std::string(what) + ": exceeds a 32-bit limit");
    case GF_ERR_LOGIC:
        throw std::logic_error(std::string(what) + ": plan exceeds the reservation bound");
    case GF_ERR_CUDA:
        throw CudaError(std::string(what) + ": CUDA error");
    default:
        throw BatchError(std::string(what) + ": device status " + std::to_string(rc));
    }
}

// ---- reservation (core/Reservation.hpp:35-71) ----
inline std::uint64_t outputChunkBound(std::uint64_t n, std::uint64_t capacity, std::uint64_t maxBins)
{
    std::uint64_t out = 0;
    throw_on(gf_output_chunk_bound(n, capacity, maxBins, &out), "outputChunkBound");
    return out;
}

inline std::uint32_t checkedOutputChunkBound(std::uint64_t n, std::uint64_t capacity, std::uint64_t maxBins)
{
    std::uint32_t out = 0;
    throw_on(gf_checked_output_chunk_bound(n, capacity, maxBins, &out), "checkedOutputChunkBound");
    return out;
}

enum class ScatterMode : std::uint32_t { SharedStaging = 0, Direct = 1 };
enum class BinPath : std::uint32_t { automatic = 0, dense = 1, hash = 2 };

// ---- optional knobs (flow/Tuning.hpp:27-145; B200 additions: fused, graphCapture, autotune) ----
struct Tuning {
    std::uint64_t seed = 0u;
    std::optional<std::uint32_t> batchChunks;      // Q
    std::optional<std::uint32_t> chunkCapacity;    // C
    std::optional<std::uint32_t> liveParticles;    // P
    std::optional<std::uint32_t> tileSize;         // particles per tile (B200 tiles)
    std::optional<std::uint32_t> numChunks;        // S
    std::optional<std::uint32_t> frameCap;
    std::optional<std::uint64_t> poolPayloadBudgetBytes;
    std::optional<ScatterMode> scatterMode;
    std::optional<BinPath> binPath;
    std::optional<std::chrono::milliseconds> stallTimeout;
    bool diagnostics = false;
    // B200: one fused classify->scan->scatter launch per partition batch instead of
    // classify + host plan + scatter.
    bool fused = true;
    // B200 runner options (results are identical either way). sinkBatchChunks: a sink may take up
    // to this many ready chunks per launch (the reference's runner takes one, GraphRunner.hpp:600;
    // at most kMaxSinkBatchChunks, independent of Q: a sink reserves no output chunks, so a
    // partition's whole fan-out can drain in one launch). multiDispatch: every idle node with ready input is dispatched in the
    // same loop iteration (the reference dispatches one node per iteration, GraphRunner.hpp:985).
    std::uint32_t sinkBatchChunks = 1u;
    bool multiDispatch = false;
    // B200: the fused partition nodes of one classifier and updater type run as one runner node
    // whose launches drain every member's ready batches (at most groupChunks input chunks, cut into
    // batches of at most Q chunks per member) in one multi-batch kernel.
    bool groupPartitions = false;
    std::uint32_t groupChunks = 1024u;
    // B200: the whole run on the device (device_flow.cuh): waves of every node's whole input as
    // one batch on one stream, chunks from a device-resident pool, one host read per wave. P, Q and
    // the runner options do not apply; partitions run the dense fused kernel.
    bool deviceResident = false;
    // B200, device-resident runs: a partition batch of at least 64 tiles and up to 64 ports runs
    // the cooperative count -> grid barrier -> scatter kernel instead of the per-tile look-back one.
    bool deviceCoop = true;
    static constexpr std::uint32_t kMaxSinkBatchChunks = 256u;

    void validate() const
    {
        auto nz = [](const auto& v, const char* name) {
            if (v.has_value() && *v == 0u)
                throw std::invalid_argument(std::string("graphflow::Tuning: ") + name + " must be non-zero");
        };
        nz(batchChunks, "batchChunks");
        nz(chunkCapacity, "chunkCapacity");
        nz(liveParticles, "liveParticles");
        nz(tileSize, "tileSize");
        nz(numChunks, "numChunks");
        nz(frameCap, "frameCap");
        nz(poolPayloadBudgetBytes, "poolPayloadBudgetBytes");
        if (groupChunks == 0u)
            throw std::invalid_argument("graphflow::Tuning: groupChunks must be non-zero");
    }
};

// ---- resolved configuration (core/Config.hpp:60-349, hot-path subset) ----
struct Config {
    static constexpr std::uint32_t denseBinLimit = 65535u;   // B200 dense path (16-bit bins)
    static constexpr std::uint32_t maxSupportedBins = 1u << 20;

    std::uint64_t numParticles = 0u;
    std::uint64_t seed = 0u;
    std::uint32_t chunkCapacity = 8192u;
    std::uint32_t liveParticles = 0u;
    std::uint32_t batchChunks = 1u;
    std::uint32_t sinkBatchChunks = 1u; // chunks per sink launch (B200 runner option)
    std::uint32_t groupChunks = 1024u;  // input chunks per partition-group launch (B200 runner option)
    std::uint32_t tileSize = 4096u;
    std::uint32_t numChunks = 0u;
    std::uint32_t maxBins = 1u;
    std::uint32_t poolOutputReserveChunks = 0u;
    ScatterMode scatterMode = ScatterMode::SharedStaging;
    BinPath binPath = BinPath::automatic;
    bool fused = true;

    BinPath effectiveBinPath() const
    {
        if (binPath != BinPath::automatic)
            return binPath;
        return maxBins > denseBinLimit ? BinPath::hash : BinPath::dense;
    }

    void validate() const
    {
        if (chunkCapacity == 0u)
            throw std::invalid_argument("graphflow::Config: chunkCapacity must be non-zero");
        if (tileSize == 0u)
            throw std::invalid_argument("graphflow::Config: tileSize must be non-zero");
        if (batchChunks == 0u)
            throw std::invalid_argument("graphflow::Config: batchChunks must be non-zero");
        if (maxBins == 0u)
            throw std::invalid_argument("graphflow::Config: maxBins must be non-zero");
        if (maxBins > maxSupportedBins)
            throw std::invalid_argument("graphflow::Config: maxBins exceeds the supported bin count");
        if (effectiveBinPath() == BinPath::dense && maxBins > denseBinLimit)
            throw std::invalid_argument("graphflow::Config: the dense bin path supports at most 65535 bins");
        if (effectiveBinPath() == BinPath::hash && scatterMode == ScatterMode::Direct)
            throw std::invalid_argument("graphflow::Config: the hash path has no direct scatter");
        if (numChunks != 0u && static_cast<std::uint64_t>(numChunks) * chunkCapacity > (1ull << 32))
            throw std::invalid_argument("graphflow::Config: numChunks * chunkCapacity exceeds 2^32 slots");
        if (numChunks != 0u && poolOutputReserveChunks >= numChunks && numParticles != 0u)
            throw std::invalid_argument("graphflow::Config: the output reserve consumes the whole pool");
    }
};

// ---- statistics (sched/GraphRunner.hpp:154-252, subset) ----
struct SchedulerStats {
    std::uint64_t completedBatches = 0u;
    std::uint64_t loopIterations = 0u;
    std::uint64_t yields = 0u;
    std::uint32_t poolChunks = 0u;
    std::uint64_t poolSlots = 0u;
    std::uint64_t poolBytes = 0u;
    std::uint32_t peakLiveChunks = 0u;
    std::uint32_t peakReservedChunks = 0u;
    std::uint32_t peakReadyChunks = 0u;
    std::uint32_t peakInflightBatches = 0u;
    std::uint64_t sourceParticles = 0u;
    std::uint64_t sourceGenerated = 0u;
    std::uint64_t sourceSunk = 0u;
    std::uint64_t sourceLiveParticles = 0u;
    std::uint32_t chunkCapacity = 0u;
    std::uint64_t kernelLaunches = 0u;
    std::uint64_t partitionBatches = 0u;
    std::uint64_t partitionLaunches = 0u; // launches that ran partition batches (a group runs many per launch)
    double setupSeconds = 0.0; // Flow::run: storage, stages and runner built
    double loopSeconds = 0.0;  // Flow::run: the scheduler loop
};

inline std::string formatSchedulerStats(const SchedulerStats& s)
{
    std::ostringstream o;
    o << "batches=" << s.completedBatches << " partitionBatches=" << s.partitionBatches
      << " partitionLaunches=" << s.partitionLaunches << " launches=" << s.kernelLaunches << " iterations=" << s.loopIterations << " yields=" << s.yields
      << " poolChunks=" << s.poolChunks << " peakLive=" << s.peakLiveChunks << " peakReserved="
      << s.peakReservedChunks << " peakReady=" << s.peakReadyChunks << " peakInflight=" << s.peakInflightBatches
      << " generated=" << s.sourceGenerated << " sunk=" << s.sourceSunk;
    return o.str();
}

// ---- chunks (core/Chunk.hpp:19-37) ----
struct ChunkHandle {
    std::uint32_t index = 0u;
    std::uint32_t generation = 0u;
    friend bool operator==(const ChunkHandle&, const ChunkHandle&) = default;
};

struct ChunkDescriptor {
    ChunkHandle handle{};
    std::uint32_t fill = 0u;
    std::uint32_t bin = 0u;
};

// Host ledger of a fixed-layout pool (core/ChunkPool.hpp, core/ChunkLedger.hpp): free list,
// per-chunk generation (stale handles are rejected), reader leases (a leased chunk cannot be
// released), and a 32-bit generation that never wraps.
class ChunkLedger {
public:
    ChunkLedger(std::uint32_t numChunks, std::uint32_t capacity)
        : m_capacity(capacity), m_generation(numChunks, 0u), m_live(numChunks, 0u), m_leases(numChunks, 0u)
    {
        if (numChunks == 0u || capacity == 0u)
            throw std::invalid_argument("graphflow::ChunkLedger: chunk count and capacity must be non-zero");
        if (static_cast<std::uint64_t>(numChunks) * capacity > (1ull << 32))
            throw std::invalid_argument("graphflow::ChunkLedger: numChunks * chunkCapacity exceeds 2^32 slots");
        for (std::uint32_t i = 0; i < numChunks; ++i)
            m_free.push_back(i);
    }

    std::uint32_t numChunks() const { return static_cast<std::uint32_t>(m_generation.size()); }
    std::uint32_t chunkCapacity() const { return m_capacity; }
    std::uint32_t freeCount() const { return static_cast<std::uint32_t>(m_free.size()); }
    std::uint32_t liveCount() const { return numChunks() - freeCount(); }
    std::uint64_t base(ChunkHandle h) const { return static_cast<std::uint64_t>(h.index) * m_capacity; }

    ChunkHandle acquire()
    {
        if (m_free.empty())
            throw BatchError("graphflow::ChunkLedger: pool exhausted");
        const std::uint32_t i = m_free.front();
        m_free.pop_front();
        m_live[i] = 1u;
        return ChunkHandle{i, m_generation[i]};
    }

    void release(ChunkHandle h)
    {
        check(h);
        if (m_leases[h.index] != 0u)
            throw std::logic_error("graphflow::ChunkLedger: releasing a leased chunk");
        if (m_generation[h.index] == std::numeric_limits<std::uint32_t>::max())
            throw std::overflow_error("graphflow::ChunkLedger: generation counter exhausted");
        ++m_generation[h.index];
        m_live[h.index] = 0u;
        m_free.push_back(h.index);
    }

    void acquireLease(ChunkHandle h)
    {
        check(h);
        ++m_leases[h.index];
    }
    void releaseLease(ChunkHandle h)
    {
        check(h);
        if (m_leases[h.index] == 0u)
            throw std::logic_error("graphflow::ChunkLedger: lease underflow");
        --m_leases[h.index];
    }
    bool valid(ChunkHandle h) const
    {
        return h.index < m_generation.size() && m_live[h.index] && m_generation[h.index] == h.generation;
    }

private:
    void check(ChunkHandle h) const
    {
        if (!valid(h))
            throw std::logic_error("graphflow::ChunkLedger: stale or foreign chunk handle");
    }
    std::uint32_t m_capacity;
    std::vector<std::uint32_t> m_generation, m_live, m_leases;
    std::deque<std::uint32_t> m_free;
};

} // namespace graphflow
