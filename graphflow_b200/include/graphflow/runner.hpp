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
// On any exception the runner drains every stream, aborts the in-flight stages, releases their
// leases and chunks and every queued chunk, then rethrows the original exception
// (GraphRunner.hpp:1173-1185).
//
// The queue operations are a policy (CudaQueueOps on the device; the scheduler's CPU tests use a
// fake), so the scheduling and failure paths are testable without a GPU.
#pragma once

#include <chrono>
#include <cstdio>
#include <deque>
#include <exception>
#include <functional>
#include <memory>
#include <optional>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime_api.h>

#include "core.hpp"
#include "stage.hpp"

namespace graphflow {

enum class NodeRole { source, transform, sink };

// Failure-injection points of the failure-path tests (the reference's FailurePoint,
// sched/GraphRunner.hpp:54-59): before a node's completion event is enqueued (item = the node's
// 1-based enqueue count), before the lease on a batch's i-th chunk is taken (item = i, 0-based),
// before a stage launch (item = the node's 1-based launch count). The hook may throw; production
// callers leave it empty.
enum class FailurePoint { eventEnqueue, leaseAcquire, launch };

// Queue operations on the CUDA device: one non-blocking stream and one completion event per node.
struct CudaQueueOps {
    using Event = cudaEvent_t;
    static void check(cudaError_t e, const char* what)
    {
        if (e != cudaSuccess)
            throw CudaError(std::string("graphflow: ") + what + ": " + cudaGetErrorString(e));
    }
    static cudaStream_t makeStream()
    {
        cudaStream_t s = nullptr;
        check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        return s;
    }
    static Event makeEvent()
    {
        cudaEvent_t e = nullptr;
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        return e;
    }
    static void destroy(cudaStream_t s, Event e) noexcept
    {
        if (e)
            cudaEventDestroy(e);
        if (s)
            cudaStreamDestroy(s);
    }
    static void record(Event e, cudaStream_t s) { check(cudaEventRecord(e, s), "cudaEventRecord"); }
    // true once the work recorded before `e` completed
    static bool done(Event e)
    {
        const cudaError_t q = cudaEventQuery(e);
        if (q == cudaErrorNotReady)
            return false;
        check(q, "cudaEventQuery");
        return true;
    }
    static void drain(cudaStream_t s) noexcept
    {
        if (s)
            cudaStreamSynchronize(s);
    }
};

template <typename Ops = CudaQueueOps>
class BasicGraphRunner {
public:
    using Event = typename Ops::Event;
    using FailureHook = std::function<void(FailurePoint, std::uint32_t node, std::uint32_t item)>;

    explicit BasicGraphRunner(ChunkLedger& ledger) : m_ledger(ledger) {}
    BasicGraphRunner(const BasicGraphRunner&) = delete;
    BasicGraphRunner& operator=(const BasicGraphRunner&) = delete;

    ~BasicGraphRunner()
    {
        for (auto& n : m_nodes)
            Ops::destroy(n.stream, n.event);
    }

    // Adds a node; `route[bin]` is the destination node index (transforms and the source), the
    // stage is owned by the caller. `tag[bin]`, when given, is written into the routed chunk's
    // descriptor bin (a partition group reads it as the member the chunk is for). Returns the node
    // index.
    std::size_t addNode(std::string name, NodeRole role, std::uint32_t bins, std::vector<int> route, Stage* stage,
                        std::vector<std::uint32_t> tag = {})
    {
        if (!tag.empty() && tag.size() != route.size())
            throw std::invalid_argument("graphflow::GraphRunner: one tag per route");
        Node n;
        n.name = std::move(name);
        n.role = role;
        n.bins = bins;
        n.route = std::move(route);
        n.tag = std::move(tag);
        n.stage = stage;
        m_nodes.push_back(std::move(n));
        Node& added = m_nodes.back();
        added.stream = Ops::makeStream();
        added.event = Ops::makeEvent();
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
    // Test hook (see FailurePoint); it runs before the injected operation and may throw.
    void setFailureHook(FailureHook hook) { m_failureHook = std::move(hook); }
    // Receives the per-node detail of a stall (names, ready lists, in-flight batches) before
    // SchedulerStallError is thrown; the exception's message holds aggregate counters only
    // (Flow.hpp:95-104).
    void setStallDetailCallback(std::function<void(const std::string&)> callback)
    {
        m_stallDetail = std::move(callback);
    }
    // Batches node k completed in the last run.
    std::uint64_t nodeCompleted(std::size_t k) const { return m_nodes.at(k).completed; }

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
                    if (!node.armed ||
                        !(node.stage->pollsCompletion() ? node.stage->completed() : Ops::done(node.event)))
                        continue;
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
                        ++node.completed;
                        // every route is checked before any output moves: an unroutable bin fails
                        // the run with the published outputs released (the inputs are still the
                        // in-flight batch's, released by the teardown)
                        for (const auto& out : outputs)
                            if (out.bin >= node.route.size() || node.route[out.bin] < 0) {
                                for (const auto& o : outputs)
                                    if (m_ledger.valid(o.handle) &&
                                        (node.role != NodeRole::source || !inputOf(*node.inflight, o.handle)))
                                        m_ledger.release(o.handle);
                                throw std::runtime_error("graphflow: node '" + node.name +
                                                         "' produced an unroutable bin");
                            }
                        for (const auto& out : outputs) {
                            ChunkDescriptor d = out;
                            if (!node.tag.empty())
                                d.bin = node.tag[out.bin];
                            m_nodes[static_cast<std::size_t>(node.route[out.bin])].ready.push_back(d);
                        }
                        if (node.role == NodeRole::sink)
                            sunk += node.inflight->particles();
                        if (node.role != NodeRole::source) {
                            for (const auto& in : node.inflight->chunks) {
                                m_ledger.releaseLease(in.handle);
                                m_ledger.release(in.handle);
                            }
                        }
                        node.leaseHeld = false;
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
                    launch(src, *m_source);
                    ++stats.kernelLaunches;
                    arm(src, *m_source);
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
                    if (std::chrono::steady_clock::now() - lastProgress > m_stallTimeout) {
                        if (m_stallDetail)
                            m_stallDetail(stallDetail());
                        throw SchedulerStallError("graphflow: scheduler stalled (generated=" +
                                                  std::to_string(generated) + " sunk=" + std::to_string(sunk) +
                                                  " free=" + std::to_string(m_ledger.freeCount()) +
                                                  " reserved=" + std::to_string(reservedTotal) + ")");
                    }
                } else {
                    idle = 0;
                    lastProgress = std::chrono::steady_clock::now();
                }
                ++stats.loopIterations;
            }
        } catch (...) {
            const std::exception_ptr original = std::current_exception();
            teardown(); // noexcept: a teardown failure must not hide the original error
            std::rethrow_exception(original);
        }
        stats.sourceGenerated = generated;
        stats.sourceSunk = sunk;
        return stats;
    }

private:
    struct Node {
        std::string name;
        NodeRole role = NodeRole::transform;
        std::uint32_t bins = 1u;
        std::vector<int> route;
        std::vector<std::uint32_t> tag;
        Stage* stage = nullptr;
        cudaStream_t stream = nullptr;
        Event event{};
        std::deque<ChunkDescriptor> ready;
        std::optional<Batch> inflight;
        bool armed = false;
        bool leaseHeld = false; // the in-flight batch's input leases are taken
        std::uint32_t reserved = 0u;
        std::uint32_t launchCount = 0u, eventEnqueues = 0u;
        std::uint64_t completed = 0u;
    };

    void arm(Node& n, std::size_t k)
    {
        ++n.eventEnqueues;
        if (m_failureHook)
            m_failureHook(FailurePoint::eventEnqueue, static_cast<std::uint32_t>(k), n.eventEnqueues);
        if (!n.stage->pollsCompletion())
            Ops::record(n.event, n.stream);
        n.armed = true;
    }
    void arm(Node& n) { arm(n, static_cast<std::size_t>(&n - m_nodes.data())); }

    std::uint32_t launch(Node& n, std::size_t k)
    {
        ++n.launchCount;
        if (m_failureHook)
            m_failureHook(FailurePoint::launch, static_cast<std::uint32_t>(k), n.launchCount);
        return n.stage->launch(n.stream, *n.inflight);
    }

    static bool inputOf(const Batch& b, ChunkHandle h)
    {
        for (const auto& c : b.chunks)
            if (c.handle == h)
                return true;
        return false;
    }

    std::string stallDetail() const
    {
        std::ostringstream o;
        for (const auto& n : m_nodes)
            o << "node '" << n.name << "': ready=" << n.ready.size() << " inflight=" << (n.inflight ? 1 : 0)
              << " armed=" << (n.armed ? 1 : 0) << " reserved=" << n.reserved << " completed=" << n.completed
              << "\n";
        return o.str();
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
        if (node.role == NodeRole::transform && node.stage->plansBatches()) {
            wanted = node.stage->planBatch(node.ready, available(), reserve);
            if (wanted == 0u || wanted > node.ready.size())
                return false;
        } else if (node.role == NodeRole::transform) {
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
        // leases on the inputs (not for a source, which owns its chunk); a failure rolls back the
        // leases taken so far and leaves the chunks in the ready list (GraphRunner.hpp:1046-1059)
        std::size_t leased = 0;
        try {
            if (node.role != NodeRole::source)
                for (std::size_t i = 0; i < batch.chunks.size(); ++i) {
                    if (m_failureHook)
                        m_failureHook(FailurePoint::leaseAcquire, static_cast<std::uint32_t>(k),
                                      static_cast<std::uint32_t>(i));
                    m_ledger.acquireLease(batch.chunks[i].handle);
                    leased = i + 1u;
                }
        } catch (...) {
            for (std::size_t i = 0; i < leased; ++i)
                m_ledger.releaseLease(batch.chunks[i].handle);
            throw;
        }
        node.inflight = std::move(batch);
        node.leaseHeld = node.role != NodeRole::source;
        node.reserved = reserve;
        reservedTotal += reserve;
        for (std::size_t i = 0; i < wanted; ++i)
            node.ready.pop_front();
        const std::uint32_t allocated = launch(node, k);
        ++stats.kernelLaunches;
        if (node.role == NodeRole::transform && node.bins > 1u) {
            stats.partitionBatches += node.stage->lastLaunchBatches();
            ++stats.partitionLaunches;
        }
        convertCredit(node, allocated, reservedTotal);
        arm(node, k);
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
            Ops::drain(n.stream);
        for (auto& n : m_nodes) {
            try {
                n.armed = false;
                if (n.inflight) {
                    n.stage->abort();
                    for (const auto& c : n.inflight->chunks) {
                        if (n.leaseHeld && m_ledger.valid(c.handle))
                            m_ledger.releaseLease(c.handle);
                        if (m_ledger.valid(c.handle))
                            m_ledger.release(c.handle);
                    }
                    n.leaseHeld = false;
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
    FailureHook m_failureHook;
    std::function<void(const std::string&)> m_stallDetail;
};

using GraphRunner = BasicGraphRunner<CudaQueueOps>;

} // namespace graphflow
