// The particle example's kernel workload on the graphflow_b200 C++ front end: Generate -> one
// partition with B ports -> one sink on every port, the partition's updater writing the chosen
// port into the record's weight, so the sorted weight histogram is the per-port occupancy.
//
// Reference (examples/particle_feedback/ in graphFlow): KernelAxes.hpp:29-42 (distributionBin:
// balanced and sparse id % B, one-hot 0, skewed id % 8 == 0 ? id % B : 0), :80-106 (classifier on
// the id, updater weight = bin), :115-167 (topology and result buffer), :169-214 (supported B,
// scatter and bin-path checks). B = 65536 (and any B with Tuning::binPath = hash) partitions
// through the per-tile hash tables.
#pragma once

#include <cstdint>

#include "particle_feedback.cuh"

namespace graphflow::particle {

enum class Distribution : std::uint32_t { balanced = 0u, oneHot = 1u, skewed = 2u, sparse = 3u };

__host__ __device__ inline std::uint32_t distributionBin(Distribution d, std::uint64_t id, std::uint32_t bins)
{
    switch (d) {
    case Distribution::oneHot:
        return 0u;
    case Distribution::skewed:
        return id % 8u == 0u ? static_cast<std::uint32_t>(id % bins) : 0u;
    default: // balanced, sparse
        return static_cast<std::uint32_t>(id % bins);
    }
}

template <std::uint32_t B>
struct KernelDistributionClassifier {
    static constexpr std::uint32_t maxBins = B;
    Distribution distribution = Distribution::balanced;
    __device__ std::uint32_t operator()(const Acc&, const Particle& p) const
    {
        return distributionBin(distribution, p.id, B);
    }
};

struct KernelBinUpdate {
    __device__ UpdateResult operator()(const Acc&, std::uint32_t bin, Particle& p) const
    {
        p.weight = bin;
        return UpdateResult::success;
    }
};

template <std::uint32_t B, typename TStorage>
SchedulerStats runKernelAxes(cuda::Device device, std::uint64_t n, Distribution distribution, Tuning tuning,
                             std::uint32_t* weights)
{
    if (n != 0u && n - 1u > rng::maxStreamId)
        throw std::overflow_error("graphflow::particle: particle count exceeds the RNG stream-id range");
    Flow<Particle, cuda::Device, TStorage> flow{device};
    auto source = flow.source("generate", GenerateParticles{});
    auto transform = flow.partition("transform", KernelDistributionClassifier<B>{distribution}, KernelBinUpdate{});
    auto sink = flow.sink("sink", RecordWeight{weights});
    flow.connect(source, transform);
    for (std::uint32_t bin = 0; bin < B; ++bin)
        flow.connect(transform, bin, sink);
    flow.configure(tuning);
    return flow.run(source, n);
}

} // namespace graphflow::particle
