// C ABI of the dense classify chain run through the C++ Flow: the kernel-level dense sweep as a
// graph of 1 to 4 chained partition nodes with the runner, pool and credits of the front end.
#include <chrono>
#include <functional>
#include <vector>

#include "gf_device_chain.cuh" // dense_chain.cuh and chain_expand_kernel

gf_status gf_flows_guard(const std::function<void()>& body); // gf_flows.cu
bool gf_runner_batched();                                       // gf_capi.cu
uint32_t gf_runner_sink_batch();
bool gf_group_partitions();                                // gf_capi.cu
bool gf_device_resident();                                 // gf_capi.cu
bool gf_device_coop();     // gf_capi.cu

namespace {

using namespace graphflow;
using namespace graphflow::dense;

template <typename TStorage>
SchedulerStats dispatchBins(std::uint32_t bins, cuda::Device device, std::uint64_t n, std::uint32_t nodes, int dist,
                            std::uint64_t seed, const double* cdf, const Tuning& t, std::uint8_t* portOf)
{
    switch (bins) {
    case 2u:
        return runDenseChain<2u, TStorage>(device, n, nodes, dist, seed, cdf, t, portOf);
    case 8u:
        return runDenseChain<8u, TStorage>(device, n, nodes, dist, seed, cdf, t, portOf);
    case 32u:
        return runDenseChain<32u, TStorage>(device, n, nodes, dist, seed, cdf, t, portOf);
    default:
        return runDenseChain<64u, TStorage>(device, n, nodes, dist, seed, cdf, t, portOf);
    }
}

} // namespace

extern "C" gf_status gf_run_dense_chain(uint64_t seed, uint64_t n, uint32_t bins, uint32_t nodes, int dist,
                                        double zipf_s, uint32_t chunk_capacity, uint32_t live_particles,
                                        uint32_t batch_chunks, int fused, int layout, uint32_t* h_port_of,
                                        gf_flow_stats* h_stats)
{
    if ((bins != 2u && bins != 8u && bins != 32u && bins != 64u) || nodes == 0u || nodes > kMaxNodes ||
        dist < GF_DIST_UNIFORM || dist > GF_DIST_ROUND_ROBIN || (dist == GF_DIST_ZIPF && !(zipf_s > 0.0)) ||
        (layout != GF_LAYOUT_SOA && layout != GF_LAYOUT_AOS))
        return GF_ERR_ARGUMENT;
    return gf_flows_guard([&] {
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::size_t m = n ? n : 1u;
        cuda::Buffer<std::uint8_t> portOf(m); // one byte per id, widened to the caller's words below
        cuda::check(cudaMemset(portOf.data(), 0xFF, m), "memset");
        cuda::Buffer<double> cdf(bins);
        if (dist == GF_DIST_ZIPF) {
            std::vector<double> h(bins);
            if (gf_zipf_cdf(zipf_s, bins, h.data()) != GF_OK)
                throw std::invalid_argument("graphflow::dense: Zipf exponent");
            cuda::check(cudaMemcpy(cdf.data(), h.data(), bins * sizeof(double), cudaMemcpyHostToDevice), "H2D");
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
        const SchedulerStats s =
            layout == GF_LAYOUT_SOA
                ? dispatchBins<SoAStorage<KeyRecord>>(bins, device, n, nodes, dist, seed, cdf.data(), t, portOf.data())
                : dispatchBins<AoSStorage<KeyRecord>>(bins, device, n, nodes, dist, seed, cdf.data(), t, portOf.data());
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (h_port_of != nullptr && n != 0u) {
            cuda::Buffer<std::uint32_t> wide(n);
            gf::chain_expand_kernel<<<static_cast<unsigned>(std::min<std::uint64_t>((n + 1023u) / 1024u, 148u * 16u)),
                                      256>>>(portOf.data(), wide.data(), n);
            cuda::check(cudaGetLastError(), "port expand launch");
            cuda::check(cudaMemcpy(h_port_of, wide.data(), n * 4u, cudaMemcpyDeviceToHost), "D2H");
        }
        if (h_stats != nullptr) {
            h_stats->completed_batches = s.completedBatches;
            h_stats->partition_batches = s.partitionBatches;
            h_stats->kernel_launches = s.kernelLaunches;
            h_stats->loop_iterations = s.loopIterations;
            h_stats->generated = s.sourceGenerated;
            h_stats->sunk = s.sourceSunk;
            h_stats->pool_chunks = s.poolChunks;
            h_stats->peak_live_chunks = s.peakLiveChunks;
            h_stats->peak_reserved_chunks = s.peakReservedChunks;
            h_stats->peak_ready_chunks = s.peakReadyChunks;
            h_stats->seconds = sec;
            h_stats->setup_seconds = s.setupSeconds;
            h_stats->loop_seconds = s.loopSeconds;
            h_stats->partition_launches = s.partitionLaunches;
        }
    });
}
