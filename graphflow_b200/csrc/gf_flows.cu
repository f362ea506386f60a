// C ABI of whole flows run through the C++ front end (Flow + GraphRunner + typed stages).
#include <chrono>
#include <functional>
#include <cstring>
#include <string>

#include "../examples/kernel_axes.cuh"
#include "../examples/particle_feedback.cuh"

namespace {

thread_local std::string g_last_error;

template <typename F>
gf_status guarded(F&& f)
{
    try {
        g_last_error.clear();
        f();
        return GF_OK;
    } catch (const graphflow::SchedulerStallError& e) {
        g_last_error = e.what();
        return GF_ERR_TIMEOUT;
    } catch (const graphflow::CudaError& e) {
        g_last_error = e.what();
        return GF_ERR_CUDA;
    } catch (const graphflow::BatchError& e) {
        g_last_error = e.what();
        return std::strstr(e.what(), "overflow") != nullptr ? GF_OVERFLOW : GF_INVALID;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return GF_ERR_ARGUMENT;
    } catch (const std::overflow_error& e) {
        g_last_error = e.what();
        return GF_ERR_RANGE;
    } catch (const std::logic_error& e) {
        g_last_error = e.what();
        return GF_ERR_LOGIC;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return GF_INVALID;
    }
}

void fill_stats(const graphflow::SchedulerStats& s, double seconds, gf_flow_stats* out)
{
    if (out == nullptr)
        return;
    out->completed_batches = s.completedBatches;
    out->partition_batches = s.partitionBatches;
    out->kernel_launches = s.kernelLaunches;
    out->loop_iterations = s.loopIterations;
    out->generated = s.sourceGenerated;
    out->sunk = s.sourceSunk;
    out->pool_chunks = s.poolChunks;
    out->peak_live_chunks = s.peakLiveChunks;
    out->peak_reserved_chunks = s.peakReservedChunks;
    out->peak_ready_chunks = s.peakReadyChunks;
    out->seconds = seconds;
    out->setup_seconds = s.setupSeconds;
    out->loop_seconds = s.loopSeconds;
    out->partition_launches = s.partitionLaunches;
}

} // namespace

bool gf_runner_batched();        // gf_capi.cu
uint32_t gf_runner_sink_batch();
bool gf_group_partitions(); // gf_capi.cu
bool gf_device_resident();  // gf_capi.cu
bool gf_device_coop();     // gf_capi.cu

// Runs a front-end call, mapping its exceptions to gf_status and the last-error message.
gf_status gf_flows_guard(const std::function<void()>& body) { return guarded(body); }
void gf_fill_flow_stats(const graphflow::SchedulerStats& s, double seconds, gf_flow_stats* out)
{
    fill_stats(s, seconds, out);
}
gf_status gf_run_particle_feedback_record_form(std::uint64_t n, std::uint32_t max_visits, graphflow::Tuning t,
                                               std::uint32_t* h_weights, std::uint32_t* h_capped,
                                               gf_flow_stats* h_stats); // gf_record_flows.cu

gf_status gf_device_policy(const gf_device_props* h_props, uint64_t n, uint32_t chunk_capacity,
                           uint32_t live_particles, uint32_t tile_size, uint32_t live_per_chunk,
                           uint64_t budget_bytes, uint64_t slot_bytes, gf_policy* h_out)
{
    if (h_out == nullptr)
        return GF_ERR_ARGUMENT;
    return guarded([&] {
        graphflow::DeviceProperties d;
        if (h_props != nullptr) {
            d.multiProcessorCount = h_props->sms;
            d.warpSize = h_props->warp_size;
            d.maxThreadsPerBlock = h_props->max_threads_per_block;
            d.maxBlocksPerGrid = h_props->max_blocks_per_grid;
            d.sharedMemPerBlockBytes = h_props->shared_mem_per_block;
            d.globalMemBytes = h_props->global_mem_bytes;
        } else {
            d = graphflow::cuda::Device::current().getDeviceProperties();
        }
        graphflow::DevicePolicyOverrides o;
        if (chunk_capacity != 0u)
            o.chunkCapacity = chunk_capacity;
        if (live_particles != 0u)
            o.liveParticles = live_particles;
        if (tile_size != 0u)
            o.tileSize = tile_size;
        graphflow::DevicePolicyConfig c;
        if (live_per_chunk != 0u)
            c.liveParticlesPerChunk = live_per_chunk;
        c.memoryBudgetBytes = budget_bytes;
        if (slot_bytes != 0u)
            c.slotBytes = slot_bytes;
        const graphflow::DevicePolicy p = graphflow::makeDevicePolicy(d, n, o, c);
        h_out->chunk_capacity = p.chunkCapacity;
        h_out->live_particles = p.liveParticles;
        h_out->tile_size = p.tileSize;
        h_out->live_explicit = p.liveParticlesExplicit ? 1u : 0u;
        h_out->budget_bytes = p.memoryBudgetBytes;
    });
}

// Records the message gf_last_error returns on this thread.
void gf_set_last_error(const char* message) { g_last_error = message != nullptr ? message : ""; }

extern "C" {

size_t gf_last_error(char* h_buf, size_t cap)
{
    if (h_buf != nullptr && cap != 0u) {
        const size_t n = g_last_error.size() < cap - 1u ? g_last_error.size() : cap - 1u;
        std::memcpy(h_buf, g_last_error.data(), n);
        h_buf[n] = '\0';
    }
    return g_last_error.size();
}

gf_status gf_run_particle_feedback(uint64_t seed, uint64_t n, uint32_t max_visits, uint32_t chunk_capacity,
                                   uint32_t live_particles, uint32_t batch_chunks, int fused, int layout,
                                   uint32_t* h_weights, uint32_t* h_capped, gf_flow_stats* h_stats)
{
    using namespace graphflow;
    using namespace graphflow::particle;
    if ((n != 0u && (h_weights == nullptr || h_capped == nullptr)) ||
        (layout != GF_LAYOUT_SOA && layout != GF_LAYOUT_AOS && layout != GF_LAYOUT_RECORD))
        return GF_ERR_ARGUMENT;
    if (layout == GF_LAYOUT_RECORD) {
        Tuning t;
        t.seed = seed;
        if (chunk_capacity != 0u)
            t.chunkCapacity = chunk_capacity;
        if (live_particles != 0u)
            t.liveParticles = live_particles;
        t.batchChunks = batch_chunks;
        t.fused = fused != 0;
        if (gf_runner_batched()) {
            t.sinkBatchChunks = gf_runner_sink_batch();
            t.multiDispatch = true;
            t.groupPartitions = gf_group_partitions();
        }
        t.deviceResident = gf_device_resident();
        t.deviceCoop = gf_device_coop();
        return gf_run_particle_feedback_record_form(n, max_visits, t, h_weights, h_capped, h_stats);
    }
    return guarded([&] {
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::size_t m = n ? n : 1u;
        cuda::Buffer<std::uint32_t> weights(m), capped(m);
        {
            std::vector<std::uint32_t> init(m, missingWeight);
            cuda::check(cudaMemcpy(weights.data(), init.data(), m * 4u, cudaMemcpyHostToDevice), "H2D");
            cuda::check(cudaMemset(capped.data(), 0, m * 4u), "memset");
        }
        Tuning t;
        t.seed = seed;
        if (chunk_capacity != 0u) // 0: the device policy derives C (and P with it)
            t.chunkCapacity = chunk_capacity;
        if (live_particles != 0u)
            t.liveParticles = live_particles;
        t.batchChunks = batch_chunks;
        t.fused = fused != 0;
        if (gf_runner_batched()) {
            t.sinkBatchChunks = gf_runner_sink_batch();
            t.multiDispatch = true;
            t.groupPartitions = gf_group_partitions();
        }
        t.deviceResident = gf_device_resident();
        t.deviceCoop = gf_device_coop();
        const auto t0 = std::chrono::steady_clock::now();
        SchedulerStats s = layout == GF_LAYOUT_SOA
                               ? runParticleFeedback<SoAStorage<Particle>>(device, n, max_visits, t, weights.data(),
                                                                           capped.data())
                               : runParticleFeedback<AoSStorage<Particle>>(device, n, max_visits, t, weights.data(),
                                                                           capped.data());
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (n != 0u) {
            cuda::check(cudaMemcpy(h_weights, weights.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
            cuda::check(cudaMemcpy(h_capped, capped.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
        }
        fill_stats(s, sec, h_stats);
    });
}

gf_status gf_run_kernel_axes(uint64_t seed, uint64_t n, uint32_t bins, int distribution, int scatter_mode,
                             int hash_path, uint32_t chunk_capacity, uint32_t live_particles, uint32_t batch_chunks,
                             int fused, uint32_t* h_weights, gf_flow_stats* h_stats)
{
    using namespace graphflow;
    using namespace graphflow::particle;
    if ((n != 0u && h_weights == nullptr) || (bins != 64u && bins != 1024u && bins != 4096u && bins != 65536u) ||
        (scatter_mode == GF_SCATTER_DIRECT && (hash_path != 0 || bins > 4096u)) ||
        distribution < GF_KDIST_BALANCED || distribution > GF_KDIST_SPARSE ||
        (scatter_mode != GF_SCATTER_SHARED && scatter_mode != GF_SCATTER_DIRECT) ||
        (distribution == GF_KDIST_SPARSE && bins < 1024u) || (scatter_mode == GF_SCATTER_DIRECT && fused != 0))
        return GF_ERR_ARGUMENT;
    return guarded([&] {
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::size_t m = n ? n : 1u;
        cuda::Buffer<std::uint32_t> weights(m);
        {
            std::vector<std::uint32_t> init(m, missingWeight);
            cuda::check(cudaMemcpy(weights.data(), init.data(), m * 4u, cudaMemcpyHostToDevice), "H2D");
        }
        Tuning t;
        t.seed = seed;
        if (chunk_capacity != 0u)
            t.chunkCapacity = chunk_capacity;
        if (live_particles != 0u)
            t.liveParticles = live_particles;
        t.batchChunks = batch_chunks;
        t.fused = fused != 0;
        t.scatterMode = scatter_mode == GF_SCATTER_DIRECT ? ScatterMode::Direct : ScatterMode::SharedStaging;
        if (hash_path != 0)
            t.binPath = BinPath::hash;
        if (gf_runner_batched()) {
            t.sinkBatchChunks = gf_runner_sink_batch();
            t.multiDispatch = true;
            t.groupPartitions = gf_group_partitions();
        }
        // device-resident runs take the fused dense partition: the fused form of the workload only
        t.deviceResident = gf_device_resident() && t.fused && hash_path == 0 && scatter_mode != GF_SCATTER_DIRECT;
        t.deviceCoop = gf_device_coop();
        const auto d = static_cast<Distribution>(distribution);
        const auto t0 = std::chrono::steady_clock::now();
        SchedulerStats s;
        if (bins == 64u)
            s = runKernelAxes<64u, SoAStorage<Particle>>(device, n, d, t, weights.data());
        else if (bins == 1024u)
            s = runKernelAxes<1024u, SoAStorage<Particle>>(device, n, d, t, weights.data());
        else if (bins == 4096u)
            s = runKernelAxes<4096u, SoAStorage<Particle>>(device, n, d, t, weights.data());
        else
            s = runKernelAxes<65536u, SoAStorage<Particle>>(device, n, d, t, weights.data());
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (n != 0u)
            cuda::check(cudaMemcpy(h_weights, weights.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
        fill_stats(s, sec, h_stats);
    });
}

gf_status gf_run_particle_feedback_kernel(uint64_t seed, uint64_t n, uint32_t max_visits, uint32_t* h_weights,
                                          uint32_t* h_capped, gf_flow_stats* h_stats)
{
    using namespace graphflow;
    using namespace graphflow::particle;
    if (n != 0u && (h_weights == nullptr || h_capped == nullptr))
        return GF_ERR_ARGUMENT;
    return guarded([&] {
        if (n != 0u && n - 1u > rng::maxStreamId)
            throw std::overflow_error("graphflow::particle: particle ids exceed the RNG stream-id range");
        if (max_visits > rng::maxStreamEvent)
            throw std::overflow_error("graphflow::particle: max visits exceeds the RNG stream-event range");
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::size_t m = n ? n : 1u;
        cuda::Buffer<std::uint32_t> weights(m), capped(m), status(1);
        std::vector<std::uint32_t> init(m, missingWeight);
        cuda::check(cudaMemcpy(weights.data(), init.data(), m * 4u, cudaMemcpyHostToDevice), "H2D");
        cuda::check(cudaMemset(capped.data(), 0, m * 4u), "memset");
        cuda::check(cudaMemset(status.data(), 0, 4u), "memset");
        const auto t0 = std::chrono::steady_clock::now();
        launchParticleTransport(nullptr, seed, 0u, n, max_visits, weights.data(), capped.data(), status.data(),
                                device.multiProcessorCount());
        cuda::check(cudaDeviceSynchronize(), "particle transport");
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::uint32_t st = 0;
        cuda::check(cudaMemcpy(&st, status.data(), 4u, cudaMemcpyDeviceToHost), "D2H");
        if (st != 0u)
            throw BatchError(std::string("particle transport: device status reports ") +
                             (st == GF_OVERFLOW ? "overflow" : "invalid"));
        if (n != 0u) {
            cuda::check(cudaMemcpy(h_weights, weights.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
            cuda::check(cudaMemcpy(h_capped, capped.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
        }
        SchedulerStats s;
        s.sourceGenerated = n;
        s.sourceSunk = n;
        s.kernelLaunches = n != 0u ? 1u : 0u;
        fill_stats(s, sec, h_stats);
    });
}

} // extern "C"
