// particle_feedback on the graphflow_b200 C++ front end: Generate -> Filter -> {A, B} -> sinks,
// with A and B feeding back into Filter.
//
// Reference (examples/particle_feedback/ in graphFlow): ParticleFunctors.hpp:33-120 (functors),
// ParticleTypes.hpp:35-47 (record {u64 id, u32 property, u32 weight, u32 visit}),
// ParticleFeedback.hpp:41-108 (topology, result buffers initialised to 0xDEADBEEF),
// ParticleTypes.hpp:206-219 (sorted weight histogram).
#pragma once

#include <cstdint>
#include <limits>

#include "graphflow/flow.cuh"

namespace graphflow::particle {

struct Particle {
    std::uint64_t id;
    std::uint32_t property;
    std::uint32_t weight;
    std::uint32_t visit;
};

} // namespace graphflow::particle

// The record's four attributes become four device columns in SoAStorage.
template <>
struct graphflow::SoAFields<graphflow::particle::Particle> {
    static constexpr std::size_t count = 4;
    template <typename P, typename F>
    __host__ __device__ static void forEach(P& p, F&& f)
    {
        f(p.id);
        f(p.property);
        f(p.weight);
        f(p.visit);
    }
};

namespace graphflow::particle {

inline constexpr std::uint32_t missingWeight = 0xDEADBEEFu;

enum class Outcome : std::uint32_t { sink = 0u, feedback = 1u, capped = 2u };

// Source: property = first draw of the source engine; record order id, property, weight, visit.
struct GenerateParticles {
    __device__ Particle operator()(const Acc&, rng::Engine& engine, std::uint64_t id) const
    {
        return Particle{id, engine(), 0u, 0u};
    }
};

// Filter: bin 1 when the filter draw reaches the particle property.
struct FilterByProperty {
    static constexpr std::uint32_t maxBins = 2u;
    __device__ std::uint32_t operator()(const Acc&, rng::Engine& engine, const Particle& p) const
    {
        return engine() >= p.property ? 1u : 0u;
    }
};

// A/B: sink, feedback, or the terminal visit cap.
struct SelectOutcome {
    static constexpr std::uint32_t maxBins = 3u;
    std::uint32_t maxVisits = 0u;
    __device__ Outcome operator()(const Acc&, rng::Engine& engine, const Particle& p) const
    {
        if (engine() < 0x80000000u)
            return Outcome::sink;
        return p.visit < maxVisits ? Outcome::feedback : Outcome::capped;
    }
};

// Feedback updater: checked weight increment and one visit.
struct UpdateWeight {
    std::uint32_t increment = 0u;
    __device__ UpdateResult operator()(const Acc&, Outcome bin, Particle& p) const
    {
        if (bin != Outcome::feedback)
            return UpdateResult::success;
        if (p.weight > std::numeric_limits<std::uint32_t>::max() - increment)
            return UpdateResult::overflow;
        p.weight += increment;
        p.visit += 1u;
        return UpdateResult::success;
    }
};

struct RecordWeight {
    std::uint32_t* weights;
    __device__ void operator()(const Acc&, const Particle& p) const { weights[p.id] = p.weight; }
};

struct RecordCapped {
    std::uint32_t* weights;
    std::uint32_t* capped;
    __device__ void operator()(const Acc&, const Particle& p) const
    {
        weights[p.id] = p.weight;
        capped[p.id] = 1u;
    }
};

// The whole feedback graph as one per-particle kernel. Each thread carries one particle from the
// source through Filter and A/B (feedback back into Filter) to its sink, calling the graph's own
// functors with the engines the Flow's stages use: node k (source 0, filter 1, A 2, B 3, sinks 4
// and 5, in the order runParticleFeedback adds them) draws from purpose 2k at the payload's
// (id, visit), its updater from 2k + 1, and the updater runs on every payload a partition emits.
// Per particle the results are therefore those of the Flow run, with no batches and no host round
// trips. Status word as the stages': overflow or invalid fail the run.
static __global__ void __launch_bounds__(256)
    particle_transport_kernel(std::uint64_t seedMixed, std::uint64_t firstId, std::uint64_t n, std::uint32_t maxVisits,
                              std::uint32_t* weights, std::uint32_t* capped, std::uint32_t* status)
{
    const GenerateParticles gen{};
    const FilterByProperty filter{};
    const SelectOutcome select{maxVisits};
    const UpdateWeight upd[2] = {UpdateWeight{1000u}, UpdateWeight{1u}};
    const RecordWeight sink{weights};
    const RecordCapped cappedSink{weights, capped};
    Status st(status);
    const Acc acc{};
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    auto generate = [&](std::uint64_t k) {
        const std::uint64_t id = firstId + k;
        rng::Engine e0 = rng::makeEngine(seedMixed, id, 0u, rng::streamPurposeForNode(0u));
        return invokeWithContext(gen, e0, st, id);
    };
    if (i >= n)
        return;
    Particle p = generate(i);
    // One visit per iteration; a lane whose particle ends starts its next particle at once, so a
    // warp stays full instead of waiting for its longest walk. Every particle's draws are keyed
    // by its own id and visit counter, so results do not depend on the order.
    for (;;) {
        rng::Engine ef = rng::engineFor(seedMixed, p, rng::streamPurposeForNode(1u));
        const std::uint32_t side = static_cast<std::uint32_t>(invokeWithContext(filter, ef, st, p));
        const std::uint32_t node = 2u + side; // A for bin 0, B for bin 1
        rng::Engine es = rng::engineFor(seedMixed, p, rng::streamPurposeForNode(node));
        const Outcome out = invokeWithContext(select, es, st, p);
        rng::Engine eu = rng::engineFor(seedMixed, p, rng::streamPurposeForNode(node, 1u));
        const std::uint32_t res = updateCode(invokeWithContext(upd[side], eu, st, out, p));
        bool done = true;
        if (res != 0u)
            gf::set_status(status, res == 1u ? GF_OVERFLOW : GF_INVALID);
        else if (out == Outcome::sink)
            sink(acc, p);
        else if (out == Outcome::capped)
            cappedSink(acc, p);
        else
            done = false;
        if (done) {
            i += stride;
            if (i >= n)
                break;
            p = generate(i);
        }
    }
}

// Enqueues the per-particle kernel for ids [firstId, firstId + n) on `stream`.
inline void launchParticleTransport(cudaStream_t stream, std::uint64_t seed, std::uint64_t firstId, std::uint64_t n,
                                    std::uint32_t maxVisits, std::uint32_t* weights, std::uint32_t* capped,
                                    std::uint32_t* status, std::uint32_t sms)
{
    if (n == 0u)
        return;
    const std::uint64_t want = (n + 255u) / 256u;
    const unsigned blocks = static_cast<unsigned>(std::min<std::uint64_t>(want, static_cast<std::uint64_t>(sms) * 16u));
    particle_transport_kernel<<<blocks, 256, 0, stream>>>(gf::mix64(seed), firstId, n, maxVisits, weights, capped,
                                                          status);
    cuda::check(cudaGetLastError(), "particle transport launch");
}

// Builds and runs the feedback graph; weights/capped are device buffers of n entries that the
// caller initialised (weights to missingWeight, capped to 0).
template <typename TStorage>
SchedulerStats runParticleFeedback(cuda::Device device, std::uint64_t n, std::uint32_t maxVisits, Tuning tuning,
                                   std::uint32_t* weights, std::uint32_t* capped)
{
    if (n != 0u && n - 1u > rng::maxStreamId)
        throw std::overflow_error("graphflow::particle: particle count exceeds the RNG stream-id range");
    if (maxVisits > rng::maxStreamEvent)
        throw std::overflow_error("graphflow::particle: max visits exceeds the RNG stream-event range");
    Flow<Particle, cuda::Device, TStorage> flow{device};
    auto source = flow.source("generate", GenerateParticles{});
    auto filter = flow.partition("filter", FilterByProperty{});
    auto processA = flow.partition("process A", SelectOutcome{maxVisits}, UpdateWeight{1000u});
    auto processB = flow.partition("process B", SelectOutcome{maxVisits}, UpdateWeight{1u});
    auto sink = flow.sink("record weight", RecordWeight{weights});
    auto cappedSink = flow.sink("record capped weight", RecordCapped{weights, capped});
    flow.connect(source, filter);
    flow.connect(filter.template out<0u>(), processA);
    flow.connect(filter.template out<1u>(), processB);
    flow.connect(processA.template out<Outcome::sink>(), sink);
    flow.connect(processB.template out<Outcome::sink>(), sink);
    flow.connect(processA.template out<Outcome::feedback>(), filter);
    flow.connect(processB.template out<Outcome::feedback>(), filter);
    flow.connect(processA.template out<Outcome::capped>(), cappedSink);
    flow.connect(processB.template out<Outcome::capped>(), cappedSink);
    flow.configure(tuning);
    return flow.run(source, n);
}

} // namespace graphflow::particle
