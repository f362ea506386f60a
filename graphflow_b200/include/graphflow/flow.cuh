// Public topology / execution API of the C++ front end, the B200 counterpart of
// graphFlow::Flow<TPayload, TDevice, TStorage> (flow/Flow.hpp:49-754 in the reference).
//
//   Flow<Particle, cuda::Device> flow{device};
//   auto src = flow.source("generate", Generate{});
//   auto filter = flow.partition("filter", Filter{});
//   auto a = flow.partition("process A", SelectOutcome{64}, UpdateWeight{1000});
//   flow.connect(src, filter);
//   flow.connect(filter.out<0>(), a);
//   ...
//   flow.configure(tuning);
//   SchedulerStats stats = flow.run(src, n);
//
// Functor shapes (flow/Concepts.hpp:126-200): an optional leading `auto const& acc`, then an
// optional `rng::Engine&`, then an optional `Status&`, then the payload: `(id)` for a source,
// `(payload const&)` returning an integral or enum bin for a classifier with
// `static constexpr maxBins`, `(bin, payload&)` returning UpdateResult (or void) for an updater,
// `(payload&)` or `(payload const&)` returning the payload or void for a transform and a sink.
#pragma once

#include <functional>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "device_flow.cuh"
#include "record.hpp"
#include "runner.hpp"
#include "stages.cuh"

namespace graphflow {

namespace detail {
struct GraphIdentity {
    std::uint64_t value;
};
inline std::uint64_t nextGraphIdentity()
{
    static std::uint64_t next = 1u;
    return next++;
}
template <typename T>
inline constexpr bool isSet = false;
template <typename... Tags>
inline constexpr bool isSet<Set<Tags...>> = true;

// A transform restricted to the attributes of TSet (flow/Flow.hpp:235-242): the functor receives
// the record as a MutableRecordProxy<TRecord, TSet> (after the usual optional accelerator,
// engine and status arguments) and changes it in place; attributes outside the set are moved
// unchanged and are out of the functor's reach at compile time.
template <typename F, typename TSet>
struct SetTransform {
    F f;
    template <typename TRecord>
    __device__ void operator()(const Acc&, rng::Engine& engine, Status& status, TRecord& p) const
    {
        auto view = p.template proxy<TSet>();
        invokeWithContext(f, engine, status, view);
    }
};

// One address per classifier and updater type pair: partition nodes that share it (and their port
// count) can run as one partition group.
template <typename TClassifier, typename TUpdate>
struct PartitionGroupKey {
    static constexpr char id = 0;
};
} // namespace detail

// flow/NodeHandle.hpp: opaque handle bound to its Flow instance.
class NodeHandle {
public:
    NodeHandle() = default;
    NodeHandle(std::shared_ptr<detail::GraphIdentity> id, std::size_t key, std::uint32_t bins, std::string name)
        : m_id(std::move(id)), m_key(key), m_bins(bins), m_name(std::move(name))
    {
    }
    std::size_t key() const { return m_key; }
    std::uint32_t bins() const { return m_bins; }
    const std::string& name() const { return m_name; }
    const std::shared_ptr<detail::GraphIdentity>& identity() const { return m_id; }

private:
    std::shared_ptr<detail::GraphIdentity> m_id;
    std::size_t m_key = 0;
    std::uint32_t m_bins = 0;
    std::string m_name;
};

using SourceHandle = NodeHandle;
using TransformHandle = NodeHandle;

// flow/Ports.hpp: one compile-time output port of a partition node.
template <std::uint32_t BinValue>
class OutputPort {
public:
    explicit OutputPort(const NodeHandle& n) : m_node(n) {}
    const NodeHandle& node() const { return m_node; }

private:
    NodeHandle m_node;
};

template <std::uint32_t MaxBins, typename TBin>
class TypedNodeHandle : public NodeHandle {
public:
    using NodeHandle::NodeHandle;
    template <auto Bin>
    OutputPort<static_cast<std::uint32_t>(Bin)> out() const
    {
        static_assert(static_cast<std::uint32_t>(Bin) < MaxBins, "graphflow: output port out of range");
        return OutputPort<static_cast<std::uint32_t>(Bin)>(*this);
    }
};

template <typename TPayload, typename TDevice = cuda::Device, typename TStorage = DefaultStorage<TPayload, TDevice>>
class Flow {
public:
    using PayloadType = TPayload;
    using Storage = TStorage;
    using Stats = SchedulerStats;

    explicit Flow(TDevice device)
        : m_device(std::move(device)),
          m_identity(std::make_shared<detail::GraphIdentity>(detail::GraphIdentity{detail::nextGraphIdentity()}))
    {
    }
    Flow(const Flow&) = delete;
    Flow& operator=(const Flow&) = delete;

    void configure(Tuning t)
    {
        t.validate();
        m_tuning = std::move(t);
    }
    const Tuning& tuning() const { return m_tuning; }

    // Flow.hpp:95-104: receives the per-node detail of a scheduler stall (node names, ready lists,
    // in-flight batches) just before SchedulerStallError is thrown; the exception's message itself
    // holds aggregate counters only.
    void setStallDetailCallback(std::function<void(const std::string&)> callback)
    {
        m_stallDetailCallback = std::move(callback);
    }

    template <typename F>
    SourceHandle source(std::string name, F f)
    {
        if (m_sourceKey)
            throw std::logic_error("graphflow: a Flow has exactly one source node");
        auto key = append(std::move(name), NodeRole::source, 1u,
                          [f](TStorage& st, const Config& c, std::uint32_t purpose) -> std::unique_ptr<Stage> {
                              return std::make_unique<SourceStage<TStorage, F>>(st, c, f, purpose);
                          });
        m_nodes[key].makeWave = [f](TStorage& st, std::uint32_t purpose) -> std::unique_ptr<devflow::WaveNode> {
            return std::make_unique<devflow::SourceWave<TStorage, F>>(st, f, purpose);
        };
        m_sourceKey = key;
        return NodeHandle(m_identity, key, 1u, m_nodes[key].name);
    }

    template <typename TClassifier, typename TUpdate = NoUpdate>
    auto partition(std::string name, TClassifier cls, TUpdate upd = {})
    {
        constexpr std::uint32_t bins = static_cast<std::uint32_t>(TClassifier::maxBins);
        static_assert(bins > 0u, "graphflow: a partition needs at least one bin");
        using TBin = ClassifierBin<TClassifier, TPayload>;
        static_assert(!std::is_void_v<TBin>, "graphflow: a classifier must return its bin (declared return type)");
        auto key = append(std::move(name), NodeRole::transform, bins,
                          [cls, upd](TStorage& st, const Config& c, std::uint32_t purpose) -> std::unique_ptr<Stage> {
                              return std::make_unique<PartitionStage<TStorage, TClassifier, TUpdate, TBin>>(
                                  st, c, cls, upd, static_cast<std::uint32_t>(TClassifier::maxBins), purpose);
                          });
        m_nodes[key].partition = true;
        m_nodes[key].makeWave = [cls, upd](TStorage& st, std::uint32_t purpose) -> std::unique_ptr<devflow::WaveNode> {
            return std::make_unique<devflow::PartitionWave<TStorage, TClassifier, TUpdate, TBin>>(
                st, cls, upd, static_cast<std::uint32_t>(TClassifier::maxBins), purpose);
        };
        m_nodes[key].groupKey = &detail::PartitionGroupKey<TClassifier, TUpdate>::id;
        m_nodes[key].makeGroup = [](TStorage& st, const Config& c, std::uint32_t b) -> std::unique_ptr<Stage> {
            using G = PartitionGroupStage<TStorage, TClassifier, TUpdate, TBin>;
            if (!G::feasible(c, b))
                return nullptr;
            return std::make_unique<G>(st, c, b);
        };
        m_nodes[key].joinGroup = [cls, upd](Stage& g, std::uint32_t purpose) -> std::uint32_t {
            return static_cast<PartitionGroupStage<TStorage, TClassifier, TUpdate, TBin>&>(g).addMember(cls, upd,
                                                                                                        purpose);
        };
        return TypedNodeHandle<bins, TBin>(m_identity, key, bins, m_nodes[key].name);
    }

    template <typename F>
    TransformHandle transform(std::string name, F f)
    {
        auto key = append(std::move(name), NodeRole::transform, 1u,
                          [f](TStorage& st, const Config& c, std::uint32_t purpose) -> std::unique_ptr<Stage> {
                              return std::make_unique<TransformStage<TStorage, F>>(st, c, f, purpose);
                          });
        m_nodes[key].makeWave = [f](TStorage& st, std::uint32_t purpose) -> std::unique_ptr<devflow::WaveNode> {
            return std::make_unique<devflow::TransformWave<TStorage, F>>(st, f, purpose);
        };
        return NodeHandle(m_identity, key, 1u, m_nodes[key].name);
    }

    template <typename TSet, typename F>
        requires detail::isSet<TSet>
    TransformHandle transform(std::string name, F f)
    {
        static_assert(isRecord<TPayload>, "graphflow: transform<Set<...>> needs a graphflow::Record payload");
        static_assert(detail::SetCompatible<TSet, typename TPayload::attribute_list>::value,
                      "graphflow: transform<Set<...>> names a tag that is not an attribute of the payload");
        return transform(std::move(name), detail::SetTransform<F, TSet>{f});
    }

    template <typename F>
    NodeHandle sink(std::string name, F f)
    {
        auto key = append(std::move(name), NodeRole::sink, 0u,
                          [f](TStorage& st, const Config& c, std::uint32_t purpose) -> std::unique_ptr<Stage> {
                              return std::make_unique<SinkStage<TStorage, F>>(st, c, f, purpose);
                          });
        m_nodes[key].makeWave = [f](TStorage& st, std::uint32_t purpose) -> std::unique_ptr<devflow::WaveNode> {
            return std::make_unique<devflow::SinkWave<TStorage, F>>(st, f, purpose);
        };
        return NodeHandle(m_identity, key, 0u, m_nodes[key].name);
    }

    void connect(const NodeHandle& from, const NodeHandle& to)
    {
        if (from.bins() != 1u)
            throw std::invalid_argument("graphflow: a multi-output node must be connected via out<Bin>()");
        connectPort(from, 0u, to);
    }
    template <std::uint32_t Bin>
    void connect(const OutputPort<Bin>& port, const NodeHandle& to)
    {
        connectPort(port.node(), Bin, to);
    }
    template <std::uint32_t MaxBins, typename TBin>
    void connect(const TypedNodeHandle<MaxBins, TBin>& from, std::uint32_t bin, const NodeHandle& to)
    {
        connectPort(from, bin, to);
    }

    // Flow.hpp:328-412: validate, resolve the configuration, build storage, stages and runner,
    // run to completion. Returns after every stream and pool chunk has been retired.
    Stats run(const NodeHandle& source, std::uint64_t itemCount)
    {
        validateForRun(source);
        if (itemCount != 0u && itemCount - 1u > rng::maxStreamId)
            throw std::overflow_error("graphflow: item count exceeds the 32 bit RNG stream-id range");
        if (m_tuning.deviceResident)
            return runDeviceResident(itemCount);
        const auto t0 = std::chrono::steady_clock::now();
        const Config config = resolveConfig(itemCount);
        m_device.makeCurrent();
        TStorage storage(m_device, config.numChunks, config.chunkCapacity);
        // partition groups: fused partition nodes of one classifier/updater type and port count run
        // as one runner node (Tuning::groupPartitions)
        const std::size_t N = m_nodes.size();
        std::vector<int> groupOf(N, -1);
        std::vector<std::uint32_t> memberOf(N, 0u);
        std::vector<std::unique_ptr<Stage>> groupStages;
        std::vector<std::vector<std::size_t>> groupMembers;
        if (m_tuning.groupPartitions)
            for (std::size_t k = 0; k < N; ++k) {
                if (!m_nodes[k].partition || groupOf[k] >= 0)
                    continue;
                std::vector<std::size_t> members;
                for (std::size_t j = k; j < N; ++j)
                    if (m_nodes[j].partition && groupOf[j] < 0 && m_nodes[j].groupKey == m_nodes[k].groupKey &&
                        m_nodes[j].bins == m_nodes[k].bins)
                        members.push_back(j);
                // a group of one still drains all of its node's ready batches per launch
                std::unique_ptr<Stage> g = m_nodes[k].makeGroup(storage, config, m_nodes[k].bins);
                if (!g)
                    continue;
                for (std::size_t j : members) {
                    memberOf[j] = m_nodes[j].joinGroup(*g, rng::streamPurposeForNode(j));
                    groupOf[j] = static_cast<int>(groupStages.size());
                }
                groupStages.push_back(std::move(g));
                groupMembers.push_back(std::move(members));
            }
        // runner node of every Flow node (a group's runner node sits at its first member)
        std::vector<std::size_t> runnerOf(N);
        std::vector<int> groupRunner(groupStages.size(), -1);
        std::size_t next = 0;
        for (std::size_t k = 0; k < N; ++k) {
            if (groupOf[k] >= 0) {
                int& r = groupRunner[static_cast<std::size_t>(groupOf[k])];
                if (r < 0)
                    r = static_cast<int>(next++);
                runnerOf[k] = static_cast<std::size_t>(r);
            } else {
                runnerOf[k] = next++;
            }
        }
        auto routeOf = [&](std::size_t k, std::vector<int>& route, std::vector<std::uint32_t>& tag) {
            for (auto r : m_nodes[k].routes) {
                route.push_back(static_cast<int>(runnerOf[r]));
                tag.push_back(groupOf[r] >= 0 ? memberOf[r] : 0u);
            }
        };
        std::vector<std::unique_ptr<Stage>> stages;
        GraphRunner runner(storage.ledger());
        for (std::size_t k = 0; k < N; ++k) {
            std::vector<int> route;
            std::vector<std::uint32_t> tag;
            if (groupOf[k] >= 0) {
                const std::size_t g = static_cast<std::size_t>(groupOf[k]);
                if (groupMembers[g].front() != k)
                    continue;
                std::string name = "group(";
                for (std::size_t j : groupMembers[g]) {
                    routeOf(j, route, tag);
                    name += (j == k ? "" : ", ") + m_nodes[j].name;
                }
                runner.addNode(name + ")", NodeRole::transform,
                               m_nodes[k].bins * static_cast<std::uint32_t>(groupMembers[g].size()), std::move(route),
                               groupStages[g].get(), std::move(tag));
                continue;
            }
            stages.push_back(m_nodes[k].make(storage, config, rng::streamPurposeForNode(k)));
            routeOf(k, route, tag);
            runner.addNode(m_nodes[k].name, m_nodes[k].role, m_nodes[k].bins, std::move(route), stages.back().get(),
                           std::move(tag));
        }
        runner.setSource(runnerOf[*m_sourceKey], itemCount, config.liveParticles);
        runner.setBatchChunks(config.batchChunks);
        runner.setSinkBatchChunks(config.sinkBatchChunks);
        runner.setMultiDispatch(m_tuning.multiDispatch);
        if (m_tuning.stallTimeout)
            runner.setStallTimeout(*m_tuning.stallTimeout);
        runner.setStallDetailCallback(m_stallDetailCallback);
        const auto t1 = std::chrono::steady_clock::now();
        Stats stats = runner.run();
        stats.setupSeconds = std::chrono::duration<double>(t1 - t0).count();
        stats.loopSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        stats.poolBytes = stats.poolSlots * TStorage::slotBytes();
        cuda::check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
        return stats;
    }

    Config resolvedConfig(std::uint64_t itemCount) const { return resolveConfig(itemCount); }

private:
    // Tuning::deviceResident (device_flow.cuh): waves of whole-list batches on one stream, chunks
    // from a device-resident pool, one read of the list counters per wave.
    Stats runDeviceResident(std::uint64_t itemCount)
    {
        using namespace devflow;
        const auto t0 = std::chrono::steady_clock::now();
        const Config config = resolveConfig(itemCount);
        if (config.effectiveBinPath() == BinPath::hash || config.scatterMode == ScatterMode::Direct)
            throw std::invalid_argument("graphflow: deviceResident runs the fused dense partition; the hash bin path "
                                        "and the direct scatter need the host runner");
        m_device.makeCurrent();
        const std::uint32_t C = config.chunkCapacity;
        const auto N = static_cast<std::uint32_t>(m_nodes.size());
        std::uint64_t sumBins = 0u;
        std::uint32_t maxBins = 1u;
        for (const auto& n : m_nodes)
            if (n.partition) {
                sumBins += n.bins;
                maxBins = std::max(maxBins, n.bins);
            }
        const std::uint64_t nIn = (itemCount + C - 1u) / C;
        const std::uint64_t S64 = 2u * (nIn + sumBins + 2u) + maxBins + 16u;
        if (S64 * C > 0xFFFFFFFFull)
            throw std::overflow_error("graphflow: the device-resident pool would exceed 2^32 slots");
        const auto S = static_cast<std::uint32_t>(S64);
        const std::uint32_t tp = (C + kTile - 1u) / kTile;
        TStorage storage(m_device, S, C);
        std::vector<std::unique_ptr<WaveNode>> waves;
        for (std::uint32_t k = 0; k < N; ++k) {
            waves.push_back(m_nodes[k].makeWave(storage, rng::streamPurposeForNode(k)));
            waves.back()->bind(k);
        }
        // routes: port b of node k feeds node routes[k][b]; one device copy of all of them
        std::vector<std::vector<std::uint32_t>> routes(N);
        std::vector<std::uint32_t> routeOffset(N, 0u), flat;
        for (std::uint32_t k = 0; k < N; ++k) {
            routeOffset[k] = static_cast<std::uint32_t>(flat.size());
            for (auto r : m_nodes[k].routes)
                routes[k].push_back(static_cast<std::uint32_t>(r));
            flat.insert(flat.end(), routes[k].begin(), routes[k].end());
        }
        cuda::Buffer<std::uint32_t> routesDev(std::max<std::size_t>(flat.size(), 1u));
        if (!flat.empty())
            cuda::check(cudaMemcpy(routesDev.data(), flat.data(), flat.size() * 4u, cudaMemcpyHostToDevice), "H2D");
        // device buffers of the run
        const std::size_t listWords = 2u * static_cast<std::size_t>(N) * S;
        cuda::Buffer<std::uint32_t> ids(listWords), fills(listWords);
        // meta: particles [2N] (u64) | counts [2N] | status, read by the host once per wave
        const std::size_t metaWords = 4u * N + 2u * N + 2u;
        cuda::Buffer<std::uint32_t> meta(metaWords);
        cuda::HostBuffer<std::uint32_t> metaHost(metaWords);
        cuda::Buffer<unsigned char> pool(gf::device_pool_bytes(S));
        const std::size_t tiles = static_cast<std::size_t>(S) * tp;
        cuda::Buffer<gf_tile> tileBuf(tiles);
        const std::uint32_t descCap = S + maxBins;
        cuda::Buffer<std::uint32_t> reserved(descCap), table(maxBins + descCap), totals(maxBins), numOut(1);
        cuda::Buffer<gf_out_desc> descs(descCap);
        cuda::Buffer<unsigned long long> portChunks(static_cast<std::size_t>(maxBins) * S);
        const std::size_t scratchBytes = 64u + tiles * maxBins * 8u;
        cuda::Buffer<unsigned char> scratch(scratchBytes);
        int sms = 1;
        {
            int dev = 0;
            cuda::check(cudaGetDevice(&dev), "cudaGetDevice");
            cuda::check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        }
        const std::uint32_t coopCtas = static_cast<std::uint32_t>(sms) * 16u;
        const std::uint64_t coopBytes =
            m_tuning.deviceCoop ? gf::any_coop_scratch_bytes(static_cast<std::uint32_t>(tiles), kTile, coopCtas) : 0u;
        cuda::Buffer<unsigned char> coopScratch(coopBytes);
        cudaStream_t s = nullptr;
        cuda::check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard()
            {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
        } guard{s};
        cuda::check(cudaMemsetAsync(meta.data(), 0, metaWords * 4u, s), "memset");
        cuda::check(cudaMemsetAsync(portChunks.data(), 0, portChunks.size() * 8u, s), "memset");
        cuda::check(cudaMemsetAsync(scratch.data(), 0, scratchBytes, s), "memset");
        auto* poolHdr = reinterpret_cast<gf::DevicePoolHdr*>(pool.data());
        gf::pool_init_kernel<<<gridFor(S, gf::kPoolThreads, 148u), gf::kPoolThreads, 0, s>>>(poolHdr, S);
        WaveContext w;
        w.s = s;
        w.pool = poolHdr;
        w.L.ids = ids.data();
        w.L.fills = fills.data();
        w.L.particles = reinterpret_cast<unsigned long long*>(meta.data());
        w.L.counts = meta.data() + 4u * N;
        w.L.N = N;
        w.L.cap = S;
        w.status = meta.data() + 6u * N;
        w.C = C;
        w.tp = tp;
        w.numChunks = S;
        w.slots = storage.slotCount();
        w.seedMixed = gf::mix64(config.seed);
        w.tiles = tileBuf.data();
        w.reserved = reserved.data();
        w.totals = totals.data();
        w.portChunks = portChunks.data();
        w.maxK = S;
        w.ctl = reinterpret_cast<gf::FusedCtl*>(scratch.data());
        w.table = table.data();
        w.descs = descs.data();
        w.descCap = descCap;
        w.numOut = numOut.data();
        w.coopScratch = coopBytes ? coopScratch.data() : nullptr;
        w.coopScratchBytes = coopBytes;
        w.coopMaxCtas = coopCtas;
        w.sms = sms;
        w.launches = 1u;
        // the wave's node order (waveOrder): a transform's successor after it where the graph allows
        std::vector<char> forwards(N, 0);
        std::vector<std::uint32_t> succ(N, kNoList), order(N, 0u);
        for (std::uint32_t k = 0; k < N; ++k) {
            forwards[k] = waves[k]->forwardsAll() ? 1 : 0;
            if (!routes[k].empty())
                succ[k] = routes[k][0];
        }
        const std::vector<std::uint32_t> seq = waveOrder(forwards, succ);
        for (std::uint32_t i = 0; i < N; ++i)
            order[seq[i]] = i;
        std::vector<std::uint32_t> waveCounts(N, 0u);
        std::vector<unsigned long long> waveParticles(N, 0u);
        std::uint32_t next = 1u;
        if (itemCount != 0u)
            waves[*m_sourceKey]->generate(w, itemCount, next, routes[*m_sourceKey][0]);
        const auto t1 = std::chrono::steady_clock::now();
        constexpr std::uint64_t kMaxWaves = 1u << 20;
        std::uint64_t wavesRun = 0u;
        for (;;) {
            cuda::check(cudaMemcpyAsync(metaHost.data(), meta.data(), metaWords * 4u, cudaMemcpyDeviceToHost, s),
                        "D2H");
            cuda::check(cudaStreamSynchronize(s), "device-resident wave");
            const std::uint32_t st = metaHost.data()[6u * N];
            if (st != 0u)
                throw BatchError("graphflow: device-resident run failed: " +
                                 std::string(st == GF_OVERFLOW ? "overflow" : statusCodeName(decodeStatus(st))) +
                                 " (code " + std::to_string(st) + ")");
            const std::uint32_t* counts = metaHost.data() + 4u * N;
            const auto* parts = reinterpret_cast<const unsigned long long*>(metaHost.data());
            bool any = false;
            for (std::uint32_t k = 0; k < N; ++k)
                any = any || counts[next * N + k] != 0u;
            if (!any)
                break;
            if (++wavesRun > kMaxWaves ||
                (m_tuning.stallTimeout && std::chrono::steady_clock::now() - t1 > *m_tuning.stallTimeout))
                throw SchedulerStallError("graphflow: device-resident run still has particles in flight after " +
                                          std::to_string(wavesRun - 1u) + " waves");
            const std::uint32_t cur = next;
            next = 1u - cur;
            // set `next` was cleared by the previous wave (or the initial memset); the first prep
            // kernel of this wave clears set `cur`, whose counters the host has just read
            w.pendingClear = cur;
            for (std::uint32_t k = 0; k < N; ++k) {
                waveCounts[k] = counts[cur * N + k];
                waveParticles[k] = parts[cur * N + k];
            }
            w.waveCounts = waveCounts.data();
            w.waveParticles = waveParticles.data();
            w.order = order.data();
            for (const std::uint32_t k : seq)
                if (waveCounts[k] != 0u)
                    waves[k]->run(w, k, waveCounts[k], waveParticles[k], cur, next, routes[k],
                                  routesDev.data() + routeOffset[k]);
        }
        gf::DevicePoolHdr hdr{};
        cuda::check(cudaMemcpyAsync(&hdr, poolHdr, sizeof(hdr), cudaMemcpyDeviceToHost, s), "D2H");
        cuda::check(cudaStreamSynchronize(s), "device-resident run");
        if (hdr.status != 0u || hdr.base != 0u)
            throw BatchError("graphflow: device-resident run ended with " + std::to_string(hdr.base) +
                             " chunks out of the pool (status " + std::to_string(hdr.status) + ")");
        Stats stats;
        stats.completedBatches = w.batches;
        stats.loopIterations = wavesRun;
        stats.poolChunks = S;
        stats.poolSlots = storage.slotCount();
        stats.poolBytes = stats.poolSlots * TStorage::slotBytes();
        stats.peakLiveChunks = hdr.peak_live;
        stats.sourceParticles = itemCount;
        stats.sourceGenerated = itemCount;
        stats.sourceSunk = w.sunk;
        stats.chunkCapacity = C;
        stats.kernelLaunches = w.launches;
        stats.partitionBatches = w.partitionBatches;
        stats.partitionLaunches = w.partitionBatches;
        stats.setupSeconds = std::chrono::duration<double>(t1 - t0).count();
        stats.loopSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        return stats;
    }

    static constexpr std::size_t kInvalid = static_cast<std::size_t>(-1);
    using Factory = std::function<std::unique_ptr<Stage>(TStorage&, const Config&, std::uint32_t)>;

    struct NodeRecord {
        std::string name;
        NodeRole role;
        std::uint32_t bins;
        std::vector<std::size_t> routes;
        Factory make;
        bool partition = false;
        const void* groupKey = nullptr; // partition nodes: classifier/updater type identity
        std::function<std::unique_ptr<Stage>(TStorage&, const Config&, std::uint32_t)> makeGroup;
        std::function<std::uint32_t(Stage&, std::uint32_t)> joinGroup;
        std::function<std::unique_ptr<devflow::WaveNode>(TStorage&, std::uint32_t)> makeWave;
    };

    std::size_t append(std::string name, NodeRole role, std::uint32_t bins, Factory make)
    {
        NodeRecord r{std::move(name), role, bins, std::vector<std::size_t>(bins, kInvalid), std::move(make)};
        m_nodes.push_back(std::move(r));
        return m_nodes.size() - 1u;
    }

    void ensureOwned(const NodeHandle& h) const
    {
        if (h.identity() != m_identity)
            throw std::invalid_argument("graphflow: the handle belongs to a different Flow instance");
        if (h.key() >= m_nodes.size())
            throw std::invalid_argument("graphflow: unknown node handle");
    }

    void connectPort(const NodeHandle& from, std::uint32_t bin, const NodeHandle& to)
    {
        ensureOwned(from);
        ensureOwned(to);
        NodeRecord& producer = m_nodes[from.key()];
        if (producer.role == NodeRole::sink)
            throw std::invalid_argument("graphflow: a sink has no outputs");
        if (bin >= producer.bins)
            throw std::invalid_argument("graphflow: output bin out of range");
        if (m_nodes[to.key()].role == NodeRole::source)
            throw std::invalid_argument("graphflow: a route may not target the source node");
        if (producer.routes[bin] != kInvalid)
            throw std::invalid_argument("graphflow: route for this output is already connected");
        producer.routes[bin] = to.key();
    }

    // Flow.hpp:525-570
    void validateForRun(const NodeHandle& source) const
    {
        ensureOwned(source);
        if (!m_sourceKey)
            throw std::logic_error("graphflow: no source node is registered");
        if (source.key() != *m_sourceKey)
            throw std::invalid_argument("graphflow: run() requires the registered source node");
        for (const auto& n : m_nodes) {
            if (n.role == NodeRole::sink)
                continue;
            for (std::size_t b = 0; b < n.routes.size(); ++b)
                if (n.routes[b] == kInvalid)
                    throw std::invalid_argument("graphflow: missing route for node '" + n.name + "' bin " +
                                                std::to_string(b));
        }
    }

    // Flow.hpp:580-626 (transform reserve, pool size) and :653-746 (resolution order).
    Config resolveConfig(std::uint64_t itemCount) const
    {
        Config c;
        c.numParticles = itemCount;
        c.seed = m_tuning.seed;
        std::uint32_t maxBins = 1u;
        for (const auto& n : m_nodes)
            maxBins = std::max(maxBins, n.bins);
        c.maxBins = maxBins;
        c.batchChunks = m_tuning.batchChunks.value_or(1u);
        c.sinkBatchChunks = std::min(std::max(m_tuning.sinkBatchChunks, 1u), Tuning::kMaxSinkBatchChunks);
        c.groupChunks = m_tuning.groupChunks;
        // C and P the caller left out come from the device policy (core/DevicePolicy.hpp:344-614)
        // with the accelerator P/C ratio of 8 and this storage's slot size, as Flow does there. The
        // payload budget is one eighth of device memory: the reference caps it at 3 GiB for 24 GB
        // devices, which on a B200 would clamp P below one chunk for records of 50 bytes and more.
        std::optional<DevicePolicy> policy;
        if (!m_tuning.chunkCapacity || !m_tuning.liveParticles) {
            const DeviceProperties props = m_device.getDeviceProperties();
            DevicePolicyConfig pc;
            pc.liveParticlesPerChunk = DevicePolicyConfig::kAcceleratorLiveParticlesPerChunk;
            pc.slotBytes = TStorage::slotBytes();
            pc.acceleratorBudgetCapBytes =
                std::max(pc.acceleratorBudgetCapBytes, props.globalMemBytes / pc.memoryBudgetDivisor);
            DevicePolicyOverrides ov;
            ov.chunkCapacity = m_tuning.chunkCapacity;
            if (ov.chunkCapacity)
                pc.maxChunkCapacity = std::max(pc.maxChunkCapacity, *ov.chunkCapacity);
            if (m_tuning.liveParticles && *m_tuning.liveParticles <= itemCount)
                ov.liveParticles = m_tuning.liveParticles;
            policy = makeDevicePolicy(props, itemCount, ov, pc);
        }
        c.chunkCapacity = m_tuning.chunkCapacity.value_or(policy ? policy->chunkCapacity : 8192u);
        c.tileSize = m_tuning.tileSize.value_or(1024u);
        c.scatterMode = m_tuning.scatterMode.value_or(ScatterMode::SharedStaging);
        c.binPath = m_tuning.binPath.value_or(BinPath::automatic);
        c.fused = m_tuning.fused;
        c.liveParticles = m_tuning.liveParticles.value_or(policy && policy->liveParticles ? policy->liveParticles : 1u);
        std::uint64_t reserve = 0;
        for (const auto& n : m_nodes)
            if (n.role == NodeRole::transform)
                reserve += checkedOutputChunkBound(c.chunkCapacity, c.chunkCapacity, n.bins);
        if (reserve > std::numeric_limits<std::uint32_t>::max())
            throw std::overflow_error("graphflow: transform output reserve exceeds 32 bits");
        c.poolOutputReserveChunks = static_cast<std::uint32_t>(reserve);
        if (m_tuning.numChunks) {
            c.numChunks = *m_tuning.numChunks;
        } else if (itemCount == 0u) {
            c.numChunks = 1u;
        } else {
            const std::uint64_t live = std::max<std::uint64_t>(1u, std::min<std::uint64_t>(c.liveParticles, itemCount));
            const std::uint64_t s = live + reserve;
            if (s > std::numeric_limits<std::uint32_t>::max())
                throw std::overflow_error("graphflow: chunk pool would exceed 2^32 chunks");
            c.numChunks = static_cast<std::uint32_t>(s);
        }
        c.validate();
        return c;
    }

    TDevice m_device;
    std::shared_ptr<detail::GraphIdentity> m_identity;
    std::optional<std::size_t> m_sourceKey;
    std::vector<NodeRecord> m_nodes;
    Tuning m_tuning;
    std::function<void(const std::string&)> m_stallDetailCallback;
};

// flow/Flow.hpp:761-762: SoA storage deduced from the payload's field list.
template <typename TPayload, typename TDevice = cuda::Device>
using SoAFlow = Flow<TPayload, TDevice, SoAStorage<TPayload, TDevice>>;

} // namespace graphflow

// The reference's namespace spelling, for callers written against graphFlow::Flow, Record, Field,
// Set and rng::StreamTraits.
namespace graphFlow = graphflow;
