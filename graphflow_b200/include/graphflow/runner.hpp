// Host scheduler of the C++ front end: one thread, one CUDA stream and event per node, no
// blocking waits in steady state.
//
// Reference (paths inside graphFlow's include/graphFlow): sched/GraphRunner.hpp:762-1171.
// Each loop iteration:
//   1. retire  - for every armed node whose event completed, advance its stage; when the batch is
//                done, route each output by node.route[bin] into the destination's ready list and
//                release the input leases and chunks (a source hands its chunk downstream);
//   2. admit   - at most one source chunk, while live particles stay below P, the remaining budget
//                allows min(C, P, remaining) particles and a free chunk exists beyond the output
//                credits already reserved;
//   3. dispatch- sinks first, then round-robin; a transform takes up to Q ready chunks and shrinks
//                the prefix until outputChunkBound(sum(fill), C, B) fits the available chunks;
//   4. stop    - source exhausted, all ready lists and in-flight batches empty, no credit left;
//   5. back off- yield after 64 idle iterations, SchedulerStallError after the stall timeout.
#pragma once

#include <chrono>
#include <deque>
#include <memory>
#include <optional>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "core.hpp"
#include "stages.cuh"

namespace graphflow {

enum class NodeRole { source, transform, sink };

class GraphRunner {
public:
    explicit GraphRunner(ChunkLedger& ledger) : m_ledger(ledger) {}
    GraphRunner(const GraphRunner&) = delete;
    GraphRunner& operator=(const GraphRunner&) = delete;

    ~GraphRunner()
    {
        for (auto& n : m_nodes) {
            if (n.event)
                cudaEventDestroy(n.event);
            if (n.stream)
                cudaStreamDestroy(n.stream);
        }
    }

    // Adds a node; `route[bin]` is the destination node index (transforms and the source), the
    // stage is owned by the caller. Returns the node index.
    std::size_t addNode(std::string name, NodeRole role, std::uint32_t bins, std::vector<int> route, Stage* stage)
    {
        Node n;
        n.name = std::move(name);
        n.role = role;
        n.bins = bins;
        n.route = std::move(route);
        n.stage = stage;
        cuda::check(cudaStreamCreateWithFlags(&n.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda::check(cudaEventCreateWithFlags(&n.event, cudaEventDisableTiming), "cudaEventCreate");
        m_nodes.push_back(std::move(n));
        return m_nodes.size() - 1u;
    }

    void setSource(std::size_t node, std::uint64_t particles, std::uint32_t liveParticles)
    {
        m_source = node;
        m_sourceParticles = particles;
        m_live = liveParticles;
    }
    void setBatchChunks(std::uint32_t q)
    {
        if (q == 0u)
            throw std::invalid_argument("graphflow::GraphRunner: batchChunks must be non-zero");
        m_Q = q;
    }
    void setStallTimeout(std::chrono::milliseconds t) { m_stallTimeout = t; }
    void setSinkBatchChunks(std::uint32_t q) { m_sinkQ = q == 0u ? 1u : q; }
    void setMultiDispatch(bool on) { m_multiDispatch = on; }

    SchedulerStats run()
    {
        if (!m_source)
            throw std::logic_error("graphflow::GraphRunner: no source node");
        SchedulerStats stats;
        stats.poolChunks = m_ledger.numChunks();
        stats.chunkCapacity = m_ledger.chunkCapacity();
        stats.poolSlots = static_cast<std::uint64_t>(m_ledger.numChunks()) * m_ledger.chunkCapacity();
        stats.sourceParticles = m_sourceParticles;
        stats.sourceLiveParticles = m_live;
        std::uint64_t generated = 0, sunk = 0;
        std::uint32_t reservedTotal = 0;
        std::uint64_t idle = 0;
        auto lastProgress = std::chrono::steady_clock::now();
        auto available = [&]() -> std::uint32_t {
            const std::uint32_t f = m_ledger.freeCount();
            return f > reservedTotal ? f - reservedTotal : 0u;
        };
        try {
            for (;;) {
                bool progress = false;
                // 1) retire
                for (std::size_t k = 0; k < m_nodes.size(); ++k) {
                    Node& node = m_nodes[k];
                    if (!node.armed)
                        continue;
                    const cudaError_t q = cudaEventQuery(node.event);
                    if (q == cudaErrorNotReady)
                        continue;
                    cuda::check(q, "cudaEventQuery");
                    node.armed = false;
                    std::uint32_t allocated = 0;
                    const bool more = node.stage->advance(node.stream, *node.inflight, allocated);
                    convertCredit(node, allocated, reservedTotal);
                    if (more) {
                        arm(node);
                    } else {
                        std::vector<ChunkDescriptor> outputs;
                        node.stage->finish(*node.inflight, outputs);
                        if (node.reserved != 0u) {
                            reservedTotal -= node.reserved;
                            node.reserved = 0u;
                        }
                        ++stats.completedBatches;
                        for (const auto& out : outputs) {
                            if (out.bin >= node.route.size() || node.route[out.bin] < 0)
                                throw std::runtime_error("graphflow: node '" + node.name + "' produced an unroutable bin");
                            m_nodes[static_cast<std::size_t>(node.route[out.bin])].ready.push_back(out);
                        }
                        if (node.role == NodeRole::sink)
                            sunk += node.inflight->particles();
                        if (node.role != NodeRole::source) {
                            for (const auto& in : node.inflight->chunks) {
                                m_ledger.releaseLease(in.handle);
                                m_ledger.release(in.handle);
                            }
                        }
                        node.inflight.reset();
                    }
                    progress = true;
                }
                observe(stats, reservedTotal);

                // 2) admit one source chunk
                Node& src = m_nodes[*m_source];
                const std::uint64_t live = generated - sunk;
                const std::uint64_t remaining = m_sourceParticles - generated;
                const std::uint64_t C = m_ledger.chunkCapacity();
                const std::uint64_t minFill =
                    m_live == 0u ? std::min(C, remaining) : std::min(std::min<std::uint64_t>(C, m_live), remaining);
                const bool enough = m_live == 0u || (live < m_live && (m_live - live) >= minFill);
                if (generated < m_sourceParticles && !src.inflight && enough && m_ledger.freeCount() > reservedTotal) {
                    std::uint64_t budget = remaining;
                    const std::uint64_t cap = m_live == 0u ? C : (m_live - live);
                    budget = std::min(std::min(budget, cap), C);
                    const ChunkHandle h = m_ledger.acquire();
                    Batch batch{{ChunkDescriptor{h, static_cast<std::uint32_t>(budget), 0u}}, generated};
                    generated += budget;
                    src.inflight = batch;
                    src.stage->launch(src.stream, *src.inflight);
                    ++stats.kernelLaunches;
                    arm(src);
                    progress = true;
                }

                // 3) dispatch: sinks first, then round-robin (one node per iteration, or every
                //    node that can take a batch with multiDispatch)
                bool dispatched = false;
                for (std::size_t k = 0; k < m_nodes.size() && (m_multiDispatch || !dispatched); ++k)
                    if (m_nodes[k].role == NodeRole::sink)
                        dispatched = tryDispatch(k, reservedTotal, available, stats) || dispatched;
                if (m_multiDispatch || !dispatched)
                    for (std::size_t j = 0; j < m_nodes.size() && (m_multiDispatch || !dispatched); ++j) {
                        const std::size_t k = (m_roundRobin + j) % m_nodes.size();
                        if (m_nodes[k].role != NodeRole::sink)
                            dispatched = tryDispatch(k, reservedTotal, available, stats) || dispatched;
                    }
                ++m_roundRobin;
                progress = progress || dispatched;
                observe(stats, reservedTotal);

                // 4) termination
                bool drained = true;
                for (const auto& n : m_nodes)
                    if (n.inflight || !n.ready.empty()) {
                        drained = false;
                        break;
                    }
                if (generated >= m_sourceParticles && drained && reservedTotal == 0u)
                    break;

                // 5) back off / stall detection
                if (!progress) {
                    if (++idle > 64u) {
                        std::this_thread::yield();
                        ++stats.yields;
                    }
                    if (std::chrono::steady_clock::now() - lastProgress > m_stallTimeout)
                        throw SchedulerStallError("graphflow: scheduler stalled (generated=" +
                                                  std::to_string(generated) + " sunk=" + std::to_string(sunk) +
                                                  " free=" + std::to_string(m_ledger.freeCount()) +
                                                  " reserved=" + std::to_string(reservedTotal) + ")");
                } else {
                    idle = 0;
                    lastProgress = std::chrono::steady_clock::now();
                }
                ++stats.loopIterations;
            }
        } catch (...) {
            teardown();
            throw;
        }
        stats.sourceGenerated = generated;
        stats.sourceSunk = sunk;
        for (const auto& n : m_nodes)
            stats.kernelLaunches += 0u;
        return stats;
    }

private:
    struct Node {
        std::string name;
        NodeRole role = NodeRole::transform;
        std::uint32_t bins = 1u;
        std::vector<int> route;
        Stage* stage = nullptr;
        cudaStream_t stream = nullptr;
        cudaEvent_t event = nullptr;
        std::deque<ChunkDescriptor> ready;
        std::optional<Batch> inflight;
        bool armed = false;
        std::uint32_t reserved = 0u;
    };

    void arm(Node& n)
    {
        cuda::check(cudaEventRecord(n.event, n.stream), "cudaEventRecord");
        n.armed = true;
    }

    void convertCredit(Node& n, std::uint32_t allocated, std::uint32_t& reservedTotal)
    {
        if (allocated == 0u)
            return;
        if (allocated > n.reserved)
            throw std::logic_error("graphflow: node acquired more chunks than reserved");
        reservedTotal -= n.reserved;
        n.reserved = 0u;
    }

    template <typename Avail>
    bool tryDispatch(std::size_t k, std::uint32_t& reservedTotal, Avail available, SchedulerStats& stats)
    {
        Node& node = m_nodes[k];
        if (node.ready.empty() || node.inflight)
            return false;
        std::size_t wanted = 1u;
        if (node.role == NodeRole::transform)
            wanted = std::min<std::size_t>(m_Q, node.ready.size());
        else if (node.role == NodeRole::sink)
            wanted = std::min<std::size_t>(m_sinkQ, node.ready.size());
        std::uint32_t reserve = 0u;
        if (node.role == NodeRole::transform) {
            std::uint64_t n = 0;
            for (std::size_t i = 0; i < wanted; ++i)
                n += node.ready[i].fill;
            while (wanted != 0u) {
                const std::uint32_t bound = checkedOutputChunkBound(n, m_ledger.chunkCapacity(), node.bins);
                if (available() >= bound) {
                    reserve = bound;
                    break;
                }
                --wanted;
                n -= node.ready[wanted].fill;
            }
            if (wanted == 0u)
                return false;
        }
        Batch batch;
        batch.chunks.assign(node.ready.begin(), node.ready.begin() + static_cast<std::ptrdiff_t>(wanted));
        for (const auto& c : batch.chunks)
            m_ledger.acquireLease(c.handle);
        node.inflight = std::move(batch);
        node.reserved = reserve;
        reservedTotal += reserve;
        for (std::size_t i = 0; i < wanted; ++i)
            node.ready.pop_front();
        const std::uint32_t allocated = node.stage->launch(node.stream, *node.inflight);
        ++stats.kernelLaunches;
        if (node.role == NodeRole::transform && node.bins > 1u)
            ++stats.partitionBatches;
        convertCredit(node, allocated, reservedTotal);
        arm(node);
        if (reservedTotal > stats.peakReservedChunks)
            stats.peakReservedChunks = reservedTotal;
        return true;
    }

    void observe(SchedulerStats& s, std::uint32_t)
    {
        std::uint32_t ready = 0, inflight = 0;
        for (const auto& n : m_nodes) {
            ready += static_cast<std::uint32_t>(n.ready.size());
            inflight += n.inflight ? 1u : 0u;
        }
        s.peakReadyChunks = std::max(s.peakReadyChunks, ready);
        s.peakInflightBatches = std::max(s.peakInflightBatches, inflight);
        s.peakLiveChunks = std::max(s.peakLiveChunks, m_ledger.liveCount());
    }

    // GraphRunner.hpp:1173-1185: drain every stream, abort stages, release leases and chunks.
    void teardown() noexcept
    {
        for (auto& n : m_nodes)
            if (n.stream)
                cudaStreamSynchronize(n.stream);
        for (auto& n : m_nodes) {
            try {
                if (n.inflight) {
                    n.stage->abort();
                    for (const auto& c : n.inflight->chunks) {
                        if (n.role != NodeRole::source)
                            m_ledger.releaseLease(c.handle);
                        if (m_ledger.valid(c.handle))
                            m_ledger.release(c.handle);
                    }
                    n.inflight.reset();
                }
                for (const auto& c : n.ready)
                    if (m_ledger.valid(c.handle))
                        m_ledger.release(c.handle);
                n.ready.clear();
            } catch (...) {
            }
        }
    }

    ChunkLedger& m_ledger;
    std::vector<Node> m_nodes;
    std::optional<std::size_t> m_source;
    std::uint64_t m_sourceParticles = 0;
    std::uint32_t m_live = 0;
    std::uint32_t m_Q = 1;
    std::uint32_t m_sinkQ = 1;
    bool m_multiDispatch = false;
    std::size_t m_roundRobin = 0;
    std::chrono::milliseconds m_stallTimeout{60000};
};

} // namespace graphflow
