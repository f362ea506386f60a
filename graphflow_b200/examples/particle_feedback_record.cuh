// particle_feedback over a named-attribute payload, the form of the reference's own example
// (examples/particle_feedback/ParticleTypes.hpp:20-47 and :226-244, ParticleFunctors.hpp:33-120):
// graphFlow::Record<Field<IdTag, u64>, Field<PropertyTag, u32>, Field<WeightTag, u32>,
// Field<VisitTag, u32>> with one device column per attribute, functors reading particle[tag],
// and the payload's RNG stream fields given by a StreamTraits specialisation. The graph, functors
// and draws are those of particle_feedback.cuh, so every particle's result is the same.
//
// Also a small graph for the attribute-subset transform (flow/Flow.hpp:235-242): Generate ->
// transform<Set<WeightTag, VisitTag>> -> sink.
#pragma once

#include <cstdint>
#include <limits>
#include <stdexcept>

#include "graphflow/flow.cuh"

namespace graphflow::particle_record {

GRAPHFLOW_TAG(Id, idTag);
GRAPHFLOW_TAG(Property, propertyTag);
GRAPHFLOW_TAG(Weight, weightTag);
GRAPHFLOW_TAG(Visit, visitTag);

using ParticleIdField = graphFlow::Field<IdTag, std::uint64_t>;
using ParticlePropertyField = graphFlow::Field<PropertyTag, std::uint32_t>;
using ParticleWeightField = graphFlow::Field<WeightTag, std::uint32_t>;
using ParticleVisitField = graphFlow::Field<VisitTag, std::uint32_t>;
using ParticleRecord =
    graphFlow::Record<ParticleIdField, ParticlePropertyField, ParticleWeightField, ParticleVisitField>;

static_assert(std::is_trivially_copyable_v<ParticleRecord>);
static_assert(std::is_default_constructible_v<ParticleRecord>);

} // namespace graphflow::particle_record

// A Record exposes no data members, so the stream fields are named explicitly.
template <>
struct graphFlow::rng::StreamTraits<graphflow::particle_record::ParticleRecord> {
    __host__ __device__ static std::uint64_t id(const graphflow::particle_record::ParticleRecord& p)
    {
        return static_cast<std::uint64_t>(p[graphflow::particle_record::idTag]);
    }
    __host__ __device__ static std::uint64_t event(const graphflow::particle_record::ParticleRecord& p)
    {
        return static_cast<std::uint64_t>(p[graphflow::particle_record::visitTag]);
    }
};

namespace graphflow::particle_record {

inline constexpr std::uint32_t missingWeight = 0xDEADBEEFu;

enum class Outcome : std::uint32_t { sink = 0u, feedback = 1u, capped = 2u };

struct GenerateParticles {
    __device__ ParticleRecord operator()(const Acc&, rng::Engine& engine, std::uint64_t id) const
    {
        return ParticleRecord{id, engine(), 0u, 0u};
    }
};

struct FilterByProperty {
    static constexpr std::uint32_t maxBins = 2u;
    __device__ std::uint32_t operator()(const Acc&, rng::Engine& engine, const ParticleRecord& p) const
    {
        return engine() >= p[propertyTag] ? 1u : 0u;
    }
};

struct SelectOutcome {
    static constexpr std::uint32_t maxBins = 3u;
    std::uint32_t maxVisits = 0u;
    __device__ Outcome operator()(const Acc&, rng::Engine& engine, const ParticleRecord& p) const
    {
        if (engine() < 0x80000000u)
            return Outcome::sink;
        return p[visitTag] < maxVisits ? Outcome::feedback : Outcome::capped;
    }
};

struct UpdateWeight {
    std::uint32_t increment = 0u;
    __device__ UpdateResult operator()(const Acc&, Outcome bin, ParticleRecord& p) const
    {
        if (bin != Outcome::feedback)
            return UpdateResult::success;
        if (p[weightTag] > std::numeric_limits<std::uint32_t>::max() - increment)
            return UpdateResult::overflow;
        p[weightTag] += increment;
        p[visitTag] += 1u;
        return UpdateResult::success;
    }
};

struct RecordWeight {
    std::uint32_t* weights;
    __device__ void operator()(const Acc&, const ParticleRecord& p) const { weights[p[idTag]] = p[weightTag]; }
};

struct RecordCapped {
    std::uint32_t* weights;
    std::uint32_t* capped;
    __device__ void operator()(const Acc&, const ParticleRecord& p) const
    {
        weights[p[idTag]] = p[weightTag];
        capped[p[idTag]] = 1u;
    }
};

// examples/particle_feedback/ParticleFeedback.hpp:41-108 over the record payload (SoA columns).
inline SchedulerStats runParticleFeedbackRecords(cuda::Device device, std::uint64_t n, std::uint32_t maxVisits,
                                                 Tuning tuning, std::uint32_t* weights, std::uint32_t* capped)
{
    if (n != 0u && n - 1u > rng::maxStreamId)
        throw std::overflow_error("graphflow::particle: particle count exceeds the RNG stream-id range");
    if (maxVisits > rng::maxStreamEvent)
        throw std::overflow_error("graphflow::particle: max visits exceeds the RNG stream-event range");
    graphFlow::SoAFlow<ParticleRecord, cuda::Device> flow{device};
    auto source = flow.source("generate", GenerateParticles{});
    auto filter = flow.partition("filter", FilterByProperty{});
    auto a = flow.partition("process A", SelectOutcome{maxVisits}, UpdateWeight{1000u});
    auto b = flow.partition("process B", SelectOutcome{maxVisits}, UpdateWeight{1u});
    auto sinkA = flow.sink("sink A", RecordWeight{weights});
    auto sinkB = flow.sink("sink B", RecordWeight{weights});
    auto capped_ = flow.sink("capped", RecordCapped{weights, capped});
    flow.connect(source, filter);
    flow.connect(filter.out<0>(), a);
    flow.connect(filter.out<1>(), b);
    flow.connect(a.out<Outcome::sink>(), sinkA);
    flow.connect(a.out<Outcome::feedback>(), filter);
    flow.connect(a.out<Outcome::capped>(), capped_);
    flow.connect(b.out<Outcome::sink>(), sinkB);
    flow.connect(b.out<Outcome::feedback>(), filter);
    flow.connect(b.out<Outcome::capped>(), capped_);
    flow.configure(tuning);
    return flow.run(source, n);
}

// A transform that sees only the weight and visit attributes of the record: weight += increment
// (wrapping), visit += 1. Reading the id or property through the proxy would not compile.
struct AddWeight {
    std::uint32_t increment;
    template <typename TProxy>
    __device__ void operator()(const Acc&, TProxy& p) const
    {
        p.template set<WeightTag>(p.template get<WeightTag>() + increment);
        p[visitTag] = p[visitTag] + 1u;
    }
};

struct RecordWeightVisit {
    std::uint32_t* weights;
    std::uint32_t* visits;
    __device__ void operator()(const Acc&, const ParticleRecord& p) const
    {
        weights[p[idTag]] = p[weightTag];
        visits[p[idTag]] = p[visitTag];
    }
};

// Generate -> transform<Set<WeightTag, VisitTag>>(AddWeight) -> sink: every particle leaves with
// weight = increment and visit = 1, its id and property untouched.
inline SchedulerStats runSetTransform(cuda::Device device, std::uint64_t n, std::uint32_t increment, Tuning tuning,
                                      std::uint32_t* weights, std::uint32_t* visits)
{
    graphFlow::SoAFlow<ParticleRecord, cuda::Device> flow{device};
    auto source = flow.source("generate", GenerateParticles{});
    auto add = flow.transform<graphFlow::Set<WeightTag, VisitTag>>("add weight", AddWeight{increment});
    auto sink = flow.sink("record", RecordWeightVisit{weights, visits});
    flow.connect(source, add);
    flow.connect(add, sink);
    flow.configure(tuning);
    return flow.run(source, n);
}

} // namespace graphflow::particle_record
