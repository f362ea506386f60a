// The kernel-level dense classify sweep through the public Flow: Generate -> NODES chained
// partition nodes -> sink, u32 keys sent to B ports. Every port of node i feeds node i + 1; the
// last node's ports all feed the sink, which records each particle's final port by id.
//
// Node i sends a key to port (key >> 8 i) mod B, so consecutive nodes re-partition the stream
// differently. Records are {u32 id, u32 key} (the particle's identity and its key); the keys are
// the ones gf_generate_keys_u32 produces for the same seed and distribution.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "graphflow/flow.cuh"

namespace graphflow::dense {

struct KeyRecord {
    std::uint32_t id;
    std::uint32_t key;
};

} // namespace graphflow::dense

template <>
struct graphflow::SoAFields<graphflow::dense::KeyRecord> {
    static constexpr std::size_t count = 2;
    template <typename P, typename F>
    __host__ __device__ static void forEach(P& p, F&& f)
    {
        f(p.id);
        f(p.key);
    }
};

namespace graphflow::dense {

inline constexpr std::uint32_t kMaxNodes = 4u;

struct GenerateKeys {
    int dist;
    std::uint64_t seedMixed;
    std::uint32_t bins;
    const double* cdf; // Zipf CDF over bins ports (device), or null
    __device__ KeyRecord operator()(const Acc&, std::uint64_t id) const
    {
        return KeyRecord{static_cast<std::uint32_t>(id), gf::synthetic_key(dist, seedMixed, id, bins, cdf)};
    }
};

template <std::uint32_t B>
struct PortOfKey {
    static constexpr std::uint32_t maxBins = B;
    std::uint32_t shift;
    __device__ std::uint32_t operator()(const Acc&, const KeyRecord& r) const { return (r.key >> shift) % B; }
};

// The port of each id as one byte (every port count here is below 255): the ids reach the sink in
// no order, and N bytes fit the 126 MB L2 at N = 1e8 where N words do not.
struct RecordPort {
    std::uint32_t shift;
    std::uint32_t bins;
    std::uint8_t* portOf;
    __device__ void operator()(const Acc&, const KeyRecord& r) const
    {
        portOf[r.id] = static_cast<std::uint8_t>((r.key >> shift) % bins);
    }
};

// Builds and runs the chain; portOf is a device buffer of n bytes.
template <std::uint32_t B, typename TStorage>
SchedulerStats runDenseChain(cuda::Device device, std::uint64_t n, std::uint32_t nodes, int dist, std::uint64_t seed,
                             const double* cdf, Tuning tuning, std::uint8_t* portOf)
{
    if (nodes == 0u || nodes > kMaxNodes)
        throw std::invalid_argument("graphflow::dense: a chain has 1 to 4 partition nodes");
    if (n != 0u && n - 1u > 0xFFFFFFFFull)
        throw std::overflow_error("graphflow::dense: particle ids are 32-bit");
    Flow<KeyRecord, cuda::Device, TStorage> flow{device};
    auto source = flow.source("generate", GenerateKeys{dist, gf::mix64(seed), B, cdf});
    using Handle = decltype(flow.partition("node", PortOfKey<B>{0u}));
    std::vector<Handle> chain;
    for (std::uint32_t i = 0; i < nodes; ++i)
        chain.push_back(flow.partition("node " + std::to_string(i), PortOfKey<B>{8u * i}));
    auto sink = flow.sink("record port", RecordPort{8u * (nodes - 1u), B, portOf});
    flow.connect(source, chain[0]);
    for (std::uint32_t i = 0; i < nodes; ++i)
        for (std::uint32_t b = 0; b < B; ++b)
            flow.connect(chain[i], b, i + 1u < nodes ? static_cast<const NodeHandle&>(chain[i + 1u]) : sink);
    flow.configure(tuning);
    return flow.run(source, n);
}

} // namespace graphflow::dense
