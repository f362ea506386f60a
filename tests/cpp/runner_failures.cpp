// CPU tests of the host scheduler's failure paths (graphflow::BasicGraphRunner) with fake stages
// and a fake queue: no device is touched. Mirrors the reference's
// tests/integration/test_failure_paths.cpp (throwing launch, failed transform batch, event-enqueue
// and lease-acquisition failures, unroutable output) and the stall detector of
// sched/GraphRunner.hpp:1153-1164. Prints one line per case and exits with the number of failures.
#include <cstdio>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "runner.hpp"

using namespace graphflow;

// Queue operations without a device: an event completes when polled unless its node is marked
// stuck (its work never finishes).
struct FakeOps {
    struct Event {
        int id = -1;
    };
    static inline std::vector<bool> stuck;
    static cudaStream_t makeStream() { return reinterpret_cast<cudaStream_t>(std::uintptr_t{0x1000u}); }
    static Event makeEvent()
    {
        stuck.push_back(false);
        return Event{static_cast<int>(stuck.size()) - 1};
    }
    static void destroy(cudaStream_t, Event) noexcept {}
    static void record(Event, cudaStream_t) {}
    static bool done(Event e) { return !stuck[static_cast<std::size_t>(e.id)]; }
    static void drain(cudaStream_t) noexcept {}
};
using Runner = BasicGraphRunner<FakeOps>;

// Source: the admitted chunk (fill = particles) goes downstream as bin 0.
struct FakeSource : Stage {
    std::function<void(std::uint64_t)> onLaunch;
    std::uint32_t launch(cudaStream_t, const Batch&) override
    {
        ++m_launches;
        if (onLaunch)
            onLaunch(m_launches);
        return 0u;
    }
    bool advance(cudaStream_t, const Batch&, std::uint32_t& a) override
    {
        a = 0u;
        return false;
    }
    void finish(const Batch& b, std::vector<ChunkDescriptor>& out) override
    {
        for (const auto& c : b.chunks)
            out.push_back(ChunkDescriptor{c.handle, c.fill, 0u});
    }
    void abort() override { ++aborts; }
    int aborts = 0;
};

// Transform: takes its output chunks (ceil(n / C), all to `bin`) at launch, from the credit the
// runner reserved; publishes them at finish, releases them on abort.
struct FakeTransform : Stage {
    ChunkLedger& ledger;
    std::uint32_t bin = 0u;
    std::function<void(std::uint64_t)> onAdvance;
    std::vector<ChunkDescriptor> pending;
    int aborts = 0;
    explicit FakeTransform(ChunkLedger& l, std::uint32_t b = 0u) : ledger(l), bin(b) {}
    std::uint32_t launch(cudaStream_t, const Batch& b) override
    {
        ++m_launches;
        std::uint64_t n = b.particles();
        const std::uint32_t C = ledger.chunkCapacity();
        const auto k = static_cast<std::uint32_t>((n + C - 1u) / C);
        for (std::uint32_t i = 0; i < k; ++i) {
            const std::uint32_t fill = n < C ? static_cast<std::uint32_t>(n) : C;
            pending.push_back(ChunkDescriptor{ledger.acquire(), fill, bin});
            n -= fill;
        }
        return k;
    }
    bool advance(cudaStream_t, const Batch&, std::uint32_t& a) override
    {
        a = 0u;
        if (onAdvance)
            onAdvance(m_launches);
        return false;
    }
    void finish(const Batch&, std::vector<ChunkDescriptor>& out) override
    {
        out.insert(out.end(), pending.begin(), pending.end());
        pending.clear();
    }
    void abort() override
    {
        ++aborts;
        for (const auto& d : pending)
            if (ledger.valid(d.handle))
                ledger.release(d.handle);
        pending.clear();
    }
};

struct FakeSink : Stage {
    std::uint64_t sunk = 0;
    int aborts = 0;
    std::uint32_t launch(cudaStream_t, const Batch& b) override
    {
        ++m_launches;
        sunk += b.particles();
        return 0u;
    }
    bool advance(cudaStream_t, const Batch&, std::uint32_t& a) override
    {
        a = 0u;
        return false;
    }
    void finish(const Batch&, std::vector<ChunkDescriptor>&) override {}
    void abort() override { ++aborts; }
};

static int g_failures = 0;
static void check(bool ok, const char* name, const std::string& why = "")
{
    std::printf("%s %s%s%s\n", ok ? "ok" : "FAIL", name, why.empty() ? "" : ": ", why.c_str());
    if (!ok)
        ++g_failures;
}

// source -> transform (2 bins: 0 -> sink, 1 -> nowhere unless `route1`) -> sink
struct Graph {
    ChunkLedger ledger;
    FakeSource src;
    FakeTransform xf;
    FakeSink sink;
    Runner runner;
    std::size_t nSrc, nXf, nSink;
    Graph(std::uint32_t chunks, std::uint32_t C, std::uint64_t particles, std::uint32_t live, std::uint32_t q = 1,
          int route1 = -1, std::uint32_t xfBin = 0)
        : ledger(chunks, C), xf(ledger, xfBin), runner(ledger)
    {
        nSrc = runner.addNode("generate", NodeRole::source, 1u, {1}, &src);
        nXf = runner.addNode("partition", NodeRole::transform, 2u, {2, route1}, &xf);
        nSink = runner.addNode("sink", NodeRole::sink, 1u, {}, &sink);
        runner.setSource(nSrc, particles, live);
        runner.setBatchChunks(q);
        runner.setStallTimeout(std::chrono::milliseconds(200));
    }
    bool restored() const { return ledger.freeCount() == ledger.numChunks(); }
};

template <typename E, typename F>
static std::string expect_throw(F f)
{
    try {
        f();
    } catch (const E& e) {
        return std::string("caught:") + e.what();
    } catch (const std::exception& e) {
        return std::string("other:") + e.what();
    }
    return "none";
}

int main()
{
    { // a normal run: every particle reaches the sink, the pool is whole again
        Graph g(16, 8, 100, 32, 2);
        SchedulerStats s = g.runner.run();
        check(g.sink.sunk == 100 && s.sourceSunk == 100 && g.restored(), "normal run drains and restores the pool");
    }
    { // a stalled device (the sink's work never completes) raises SchedulerStallError; the
      // detail callback gets the per-node state, the message holds aggregate counters only
        Graph g(16, 8, 100, 32);
        FakeOps::stuck[static_cast<std::size_t>(g.nSink) + FakeOps::stuck.size() - 3u] = true;
        std::string detail;
        g.runner.setStallDetailCallback([&](const std::string& d) { detail = d; });
        const std::string r = expect_throw<SchedulerStallError>([&] { g.runner.run(); });
        check(r.rfind("caught:graphflow: scheduler stalled", 0) == 0, "stall raises SchedulerStallError", r);
        check(detail.find("node 'sink'") != std::string::npos && r.find("sink") == std::string::npos,
              "stall detail goes to the callback, not the message", detail);
        check(g.restored() && g.sink.aborts == 1, "stall teardown releases every chunk and aborts the sink");
        FakeOps::stuck.assign(FakeOps::stuck.size(), false);
    }
    { // a throwing source launch fails the run with that error, not a stall
        Graph g(16, 8, 100, 8);
        g.src.onLaunch = [](std::uint64_t k) {
            if (k == 2u)
                throw BatchError("source launch failed on purpose");
        };
        const std::string r = expect_throw<BatchError>([&] { g.runner.run(); });
        check(r == "caught:source launch failed on purpose", "throwing source launch surfaces its error", r);
        check(g.restored(), "throwing source launch restores the pool");
    }
    { // a failed transform batch (advance throws) aborts the stage and releases leases and outputs
        Graph g(16, 8, 100, 32, 2);
        g.xf.onAdvance = [](std::uint64_t k) {
            if (k == 3u)
                throw BatchError("transform status rejected");
        };
        const std::string r = expect_throw<BatchError>([&] { g.runner.run(); });
        check(r == "caught:transform status rejected", "throwing advance surfaces its error", r);
        check(g.restored() && g.xf.aborts == 1 && g.xf.pending.empty(), "throwing advance releases leases and outputs");
    }
    { // lease acquisition fails on the second chunk of a batch: the first lease is rolled back
        Graph g(16, 8, 100, 64, 4);
        int calls = 0;
        g.runner.setFailureHook([&](FailurePoint p, std::uint32_t node, std::uint32_t item) {
            if (p == FailurePoint::leaseAcquire && node == g.nXf && item == 1u && ++calls == 1)
                throw BatchError("lease refused");
        });
        const std::string r = expect_throw<BatchError>([&] { g.runner.run(); });
        check(r == "caught:lease refused", "lease failure surfaces its error", r);
        check(g.restored(), "lease failure rolls back the leases taken and restores the pool");
    }
    { // the completion event of a planned transform batch cannot be enqueued
        Graph g(16, 8, 100, 32, 2);
        g.runner.setFailureHook([&](FailurePoint p, std::uint32_t node, std::uint32_t item) {
            if (p == FailurePoint::eventEnqueue && node == g.nXf && item == 2u)
                throw CudaError("event enqueue failed on purpose");
        });
        const std::string r = expect_throw<CudaError>([&] { g.runner.run(); });
        check(r == "caught:event enqueue failed on purpose", "event enqueue failure surfaces its error", r);
        check(g.restored() && g.xf.aborts == 1, "event enqueue failure releases the planned batch");
    }
    { // a stage launch refused by the hook (the reference's chunkLaunch point)
        Graph g(16, 8, 100, 32, 2);
        g.runner.setFailureHook([&](FailurePoint p, std::uint32_t node, std::uint32_t item) {
            if (p == FailurePoint::launch && node == g.nSink && item == 1u)
                throw BatchError("sink launch refused");
        });
        const std::string r = expect_throw<BatchError>([&] { g.runner.run(); });
        check(r == "caught:sink launch refused" && g.restored(), "refused launch restores the pool", r);
    }
    { // an output to a bin with no route fails the run and still releases the batch input
        Graph g(16, 8, 100, 32, 1, -1, 1u);
        const std::string r = expect_throw<std::runtime_error>([&] { g.runner.run(); });
        check(r.find("unroutable") != std::string::npos && g.restored(), "unroutable output releases the input", r);
    }
    std::printf("%d failures\n", g_failures);
    return g_failures;
}
