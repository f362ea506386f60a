// Typed kernels of the C++ front end (source, transform, sink) and the adapters that run user
// classifiers and updaters inside the partition kernels of gf_partition.cuh / gf_hash.cuh.
//
// Reference (paths inside graphFlow's include/graphFlow): flow/Execution.hpp:665-692
// (SourceKernel), :694-776 (TransformKernel: out-of-place copy-with-functor, output position =
// dense concatenation of the batch), :1509-1534 (SinkKernel), :870-1189 (typed partition kernels:
// classifier engine purpose p, updater purpose p + 1, both keyed by the loaded payload).
#pragma once

#include "device.cuh"
#include "gf_partition.cuh"

namespace graphflow {

// Host-polled completion of a front-end kernel: the launch's last CTA copies the status word into
// a record in mapped host memory ([0] sequence, [1] status), clears the status word and the CTA
// counter for the next launch, and writes the sequence number last, so the host reads a complete
// record with a plain load and needs neither a copy nor an event.
struct Completion {
    std::uint32_t* ctas = nullptr; // device counter of retired CTAs, zero between launches
    std::uint32_t* rec = nullptr;  // mapped host record
    std::uint32_t seq = 0u;
};

__device__ inline void complete(const Completion& c, std::uint32_t* status)
{
    if (c.rec == nullptr)
        return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(c.ctas, 1u) + 1u == gridDim.x) {
            *c.ctas = 0u;
            __threadfence(); // every other CTA's status write came before its count
            c.rec[1] = gf::ld_relaxed_u32(status);
            *status = 0u;
            __threadfence_system();
            *reinterpret_cast<volatile std::uint32_t*>(c.rec) = c.seq;
        }
    }
}

// One <= tile slice of one input chunk with its position in the batch's dense output.
struct MoveTile {
    std::uint32_t in_chunk;
    std::uint32_t in_offset;
    std::uint32_t count;
    std::uint32_t out_pos;
};

template <typename TFunctor, typename TView>
__global__ void __launch_bounds__(256) source_kernel(TFunctor f, TView view, std::uint64_t seed_mixed,
                                                     std::uint32_t purpose, std::uint64_t first_id,
                                                     std::uint64_t base, std::uint32_t fill, std::uint32_t* status,
                                                     Completion done = {})
{
    for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < fill; i += gridDim.x * blockDim.x) {
        const std::uint64_t id = first_id + i;
        rng::Engine engine = rng::makeEngine(seed_mixed, id, 0u, purpose);
        Status st(status);
        auto payload = invokeWithContext(f, engine, st, id);
        view.store(base + i, static_cast<typename TView::Payload>(payload));
    }
    complete(done, status);
}

// Out-of-place transform over a batch: input item i of tile t goes to dense output position
// tile.out_pos + i, i.e. output chunk out_chunks[pos / C] at offset pos % C.
template <typename TFunctor, typename TView>
__global__ void __launch_bounds__(256) transform_kernel(TFunctor f, TView view, std::uint64_t seed_mixed,
                                                        std::uint32_t purpose, const MoveTile* tiles,
                                                        std::uint32_t n_tiles, const std::uint32_t* out_chunks,
                                                        std::uint32_t n_out, std::uint32_t capacity, gf::FastDiv fdc,
                                                        std::uint64_t slots, std::uint32_t* status,
                                                        Completion done = {})
{
    for (std::uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const MoveTile tile = tiles[t];
        const std::uint64_t in_base = static_cast<std::uint64_t>(tile.in_chunk) * capacity + tile.in_offset;
        for (std::uint32_t i = threadIdx.x; i < tile.count; i += blockDim.x) {
            const std::uint32_t pos = tile.out_pos + i;
            const std::uint32_t k = fdc.div(pos);
            if (k >= n_out) {
                gf::set_status(status, GF_OVERFLOW);
                continue;
            }
            const std::uint64_t out = static_cast<std::uint64_t>(out_chunks[k]) * capacity + (pos - k * capacity);
            if (in_base + i >= slots || out >= slots) {
                gf::set_status(status, GF_INVALID);
                continue;
            }
            auto p = view.load(in_base + i);
            rng::Engine engine = rng::engineFor(seed_mixed, p, purpose);
            Status st(status);
            applyTransform(f, engine, st, p);
            view.store(out, p);
        }
    }
    complete(done, status);
}

// Sink over a batch of input chunks (the reference launches one per chunk).
template <typename TFunctor, typename TView>
__global__ void __launch_bounds__(256) sink_kernel(TFunctor f, TView view, std::uint64_t seed_mixed,
                                                   std::uint32_t purpose, const MoveTile* tiles,
                                                   std::uint32_t n_tiles, std::uint32_t capacity,
                                                   std::uint64_t slots, std::uint32_t* status, Completion done = {})
{
    for (std::uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const MoveTile tile = tiles[t];
        const std::uint64_t in_base = static_cast<std::uint64_t>(tile.in_chunk) * capacity + tile.in_offset;
        for (std::uint32_t i = threadIdx.x; i < tile.count; i += blockDim.x) {
            if (in_base + i >= slots) {
                gf::set_status(status, GF_INVALID);
                continue;
            }
            const auto p = view.load(in_base + i);
            rng::Engine engine = rng::engineFor(seed_mixed, p, purpose);
            Status st(status);
            invokeWithContext(f, engine, st, p);
        }
    }
    complete(done, status);
}

// Storage view as a partition-kernel access policy (same columns in and out: the batch reads
// its input chunks and writes distinct output chunks).
template <typename TView>
struct ViewAccess {
    using Payload = typename TView::Payload;
    TView view;
    __device__ Payload load(std::uint64_t s) const { return view.load(s); }
    __device__ void store(std::uint64_t s, const Payload& p) const { view.store(s, p); }
};

// User classifier inside the partition kernels: engine at (id, event, purpose) of the loaded
// payload, optional status; the result is the bin (enum or integral).
template <typename TClassifier, typename P>
struct ClassifyAdapter {
    TClassifier f;
    std::uint64_t seed_mixed;
    std::uint32_t purpose;
    std::uint32_t* status;
    __device__ std::uint32_t operator()(const P& p) const
    {
        rng::Engine engine = rng::engineFor(seed_mixed, p, purpose);
        Status st(status);
        return static_cast<std::uint32_t>(invokeWithContext(f, engine, st, p));
    }
};

// User updater inside the scatter: engine at purpose + 1 of the loaded payload, applied once per
// emitted payload; returns the UpdateResult code the kernels expect.
template <typename TUpdate, typename TBin, typename P>
struct UpdateAdapter {
    TUpdate f;
    std::uint32_t purpose;
    std::uint32_t* status;
    __device__ std::uint32_t operator()(std::uint32_t bin, P& p, std::uint64_t seed_mixed) const
    {
        rng::Engine engine = rng::engineFor(seed_mixed, p, purpose);
        Status st(status);
        return updateCode(invokeWithContext(f, engine, st, static_cast<TBin>(bin), p));
    }
};

} // namespace graphflow
