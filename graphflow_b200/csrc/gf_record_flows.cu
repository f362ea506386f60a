// Flow entry points over named-attribute payloads (graphFlow::Record): particle_feedback in the
// reference example's own payload form, and the attribute-subset transform graph.
#include <chrono>
#include <functional>
#include <vector>

#include "../examples/particle_feedback_record.cuh"

gf_status gf_flows_guard(const std::function<void()>& body); // gf_flows.cu
void gf_fill_flow_stats(const graphflow::SchedulerStats& s, double seconds, gf_flow_stats* out); // gf_flows.cu

// Called by gf_run_particle_feedback for GF_LAYOUT_RECORD, with the caller's validated arguments
// and the tuning it resolved.
gf_status gf_run_particle_feedback_record_form(std::uint64_t n, std::uint32_t max_visits, graphflow::Tuning t,
                                               std::uint32_t* h_weights, std::uint32_t* h_capped,
                                               gf_flow_stats* h_stats)
{
    using namespace graphflow;
    using namespace graphflow::particle_record;
    return gf_flows_guard([&] {
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::size_t m = n ? n : 1u;
        cuda::Buffer<std::uint32_t> weights(m), capped(m);
        {
            std::vector<std::uint32_t> init(m, missingWeight);
            cuda::check(cudaMemcpy(weights.data(), init.data(), m * 4u, cudaMemcpyHostToDevice), "H2D");
            cuda::check(cudaMemset(capped.data(), 0, m * 4u), "memset");
        }
        const auto t0 = std::chrono::steady_clock::now();
        const SchedulerStats s = runParticleFeedbackRecords(device, n, max_visits, t, weights.data(), capped.data());
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (n != 0u) {
            cuda::check(cudaMemcpy(h_weights, weights.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
            cuda::check(cudaMemcpy(h_capped, capped.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
        }
        gf_fill_flow_stats(s, sec, h_stats);
    });
}

bool gf_device_resident(); // gf_capi.cu
bool gf_device_coop();     // gf_capi.cu

extern "C" gf_status gf_run_set_transform(uint64_t seed, uint64_t n, uint32_t increment, uint32_t chunk_capacity,
                                          uint32_t live_particles, uint32_t batch_chunks, uint32_t* h_weights,
                                          uint32_t* h_visits, gf_flow_stats* h_stats)
{
    using namespace graphflow;
    using namespace graphflow::particle_record;
    if (n != 0u && (h_weights == nullptr || h_visits == nullptr))
        return GF_ERR_ARGUMENT;
    return gf_flows_guard([&] {
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::size_t m = n ? n : 1u;
        cuda::Buffer<std::uint32_t> weights(m), visits(m);
        cuda::check(cudaMemset(weights.data(), 0xFF, m * 4u), "memset");
        cuda::check(cudaMemset(visits.data(), 0xFF, m * 4u), "memset");
        Tuning t;
        t.seed = seed;
        if (chunk_capacity != 0u)
            t.chunkCapacity = chunk_capacity;
        if (live_particles != 0u)
            t.liveParticles = live_particles;
        t.batchChunks = batch_chunks;
        t.deviceResident = gf_device_resident();
        t.deviceCoop = gf_device_coop();
        const auto t0 = std::chrono::steady_clock::now();
        const SchedulerStats s = runSetTransform(device, n, increment, t, weights.data(), visits.data());
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (n != 0u) {
            cuda::check(cudaMemcpy(h_weights, weights.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
            cuda::check(cudaMemcpy(h_visits, visits.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
        }
        gf_fill_flow_stats(s, sec, h_stats);
    });
}
