// C ABI of the photon_scattering transform bodies: the graph through the C++ Flow, or the fused
// per-photon transport kernel over the same functors.
#include <chrono>
#include <functional>
#include <cstring>
#include <string>
#include <vector>

#include "../examples/photon.cuh"

gf_status gf_flows_guard(const std::function<void()>& body); // gf_flows.cu
bool gf_runner_batched();                                       // gf_capi.cu
uint32_t gf_runner_sink_batch();                                // gf_capi.cu

bool gf_group_partitions(); // gf_capi.cu
bool gf_device_resident();  // gf_capi.cu
bool gf_device_coop();     // gf_capi.cu

namespace {

using namespace graphflow;
using namespace graphflow::photon;

// Path trace of ids [0, ids) with up to `vertices` vertices each; ids = 0 traces nothing.
struct TraceRequest {
    std::uint64_t ids = 0u;
    std::uint32_t vertices = 0u;
    gf_trace_vertex* hVertices = nullptr;
    std::uint32_t* hCounts = nullptr;
    std::uint32_t* hTruncated = nullptr;
};

template <typename T>
void runTyped(std::uint64_t seed, std::uint64_t firstId, std::uint64_t n, const gf_photon_params& P, int exec,
              std::uint32_t C, std::uint32_t live, std::uint32_t Q, uint32_t* hEvent, uint32_t* hSc, double* hW,
              double* hCos, double* hPos, double* hDir, double* hRefl, double* hTrans, uint64_t* hCounts,
              gf_flow_stats* hStats, const TraceRequest& tr = {})
{
    if (exec == GF_EXEC_FLOW && firstId != 0u)
        throw std::invalid_argument("graphflow::photon: a Flow run starts at id 0");
    cuda::Device device = cuda::Device::current();
    device.makeCurrent();
    const std::size_t m = n ? n : 1u;
    const bool wantRecords = hEvent || hSc || hW || hCos || hPos || hDir;
    cuda::Buffer<TerminalT<T>> records(wantRecords ? m : 1u);
    cuda::Buffer<std::uint32_t> visits(m);
    const std::uint32_t hb = P.model == GF_PHOTON_WEIGHTED ? P.hist_bins : 0u;
    cuda::Buffer<T> refl(hb ? hb : 1u), trans(hb ? hb : 1u);
    cuda::Buffer<unsigned long long> counts(5);
    cuda::Buffer<std::uint32_t> status(1);
    cuda::check(cudaMemset(visits.data(), 0, m * 4u), "memset");
    cuda::check(cudaMemset(refl.data(), 0, sizeof(T) * (hb ? hb : 1u)), "memset");
    cuda::check(cudaMemset(trans.data(), 0, sizeof(T) * (hb ? hb : 1u)), "memset");
    cuda::check(cudaMemset(counts.data(), 0, 40), "memset");
    cuda::check(cudaMemset(status.data(), 0, 4), "memset");
    if (wantRecords)
        cuda::check(cudaMemset(records.data(), 0xFF, sizeof(TerminalT<T>) * m), "memset");

    const SlabT<T> slab{static_cast<T>(P.thickness), static_cast<T>(P.sigma_s), static_cast<T>(P.sigma_a)};
    const std::size_t traceSlots = static_cast<std::size_t>(tr.ids) * tr.vertices;
    cuda::Buffer<TraceVertexT<T>> traceVertices(traceSlots);
    cuda::Buffer<std::uint32_t> traceCounts(tr.ids), traceTruncated(tr.ids);
    if (tr.ids != 0u) {
        cuda::check(cudaMemset(traceCounts.data(), 0, 4u * tr.ids), "memset");
        cuda::check(cudaMemset(traceTruncated.data(), 0, 4u * tr.ids), "memset");
    }
    SchedulerStats stats;
    const auto t0 = std::chrono::steady_clock::now();
    auto run = [&](auto propose, auto scatter, auto terminal) {
        if (exec == GF_EXEC_FLOW) {
            Tuning t;
            t.seed = seed;
            if (C != 0u) // 0: the device policy derives C (and P with it)
                t.chunkCapacity = C;
            if (live != 0u)
                t.liveParticles = live;
            t.batchChunks = Q;
            if (gf_runner_batched()) {
                t.sinkBatchChunks = gf_runner_sink_batch();
                t.multiDispatch = true;
                t.groupPartitions = gf_group_partitions();
            }
            t.deviceResident = gf_device_resident();
            t.deviceCoop = gf_device_coop();
            stats = runPhotonFlow<T, SoAStorage<PhotonT<T>>>(device, n, propose, slab, scatter, terminal, t);
        } else if (n != 0u) {
            const unsigned blocks = static_cast<unsigned>(std::min<std::uint64_t>((n + 255u) / 256u, 148u * 64u));
            transport_kernel<T><<<blocks, 256>>>(propose, AdvanceToEventT<T>{slab}, scatter, terminal,
                                                 gf::mix64(seed), firstId, n, status.data());
            cuda::check(cudaGetLastError(), "transport launch");
            cuda::check(cudaDeviceSynchronize(), "transport");
        }
    };
    // an untraced run instantiates the functors without trace code (NoTraceT)
    auto withTrace = [&](auto trace) {
        using Tr = decltype(trace);
        const RecordTerminalT<T, Tr> terminal{wantRecords ? records.data() : nullptr,
                                              visits.data(),
                                              refl.data(),
                                              trans.data(),
                                              hb,
                                              counts.data(),
                                              trace};
        if (P.model == GF_PHOTON_ANALOG)
            run(ProposeFlightT<T>{slab, P.max_scatters}, ScatterT<T, Tr>{P.isotropic != 0, trace}, terminal);
        else
            run(ProposeWeightedT<T>{slab,
                                    WeightedT<T>{static_cast<T>(P.g), static_cast<T>(P.roulette_threshold),
                                                 static_cast<T>(P.roulette_survival)},
                                    P.max_scatters},
                ScatterHGT<T, Tr>{static_cast<T>(P.g), trace}, terminal);
    };
    if (tr.ids != 0u)
        withTrace(TraceT<T>{traceVertices.data(), traceCounts.data(), traceTruncated.data(), tr.vertices, tr.ids});
    else
        withTrace(NoTraceT<T>{});
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::uint32_t st = 0;
    cuda::check(cudaMemcpy(&st, status.data(), 4, cudaMemcpyDeviceToHost), "D2H");
    if (st != 0u)
        throw BatchError("photon transport: device status reports " + std::to_string(st));
    std::vector<std::uint32_t> v(m);
    cuda::check(cudaMemcpy(v.data(), visits.data(), m * 4u, cudaMemcpyDeviceToHost), "D2H");
    for (std::uint64_t i = 0; i < n; ++i)
        if (v[i] != 1u)
            throw BatchError("photon transport: photon " + std::to_string(firstId + i) +
                             " did not reach the terminal exactly once");
    if (wantRecords && n) {
        std::vector<TerminalT<T>> r(n);
        cuda::check(cudaMemcpy(r.data(), records.data(), sizeof(TerminalT<T>) * n, cudaMemcpyDeviceToHost), "D2H");
        for (std::uint64_t i = 0; i < n; ++i) {
            if (hEvent)
                hEvent[i] = r[i].event;
            if (hSc)
                hSc[i] = r[i].scatterCount;
            if (hW)
                hW[i] = static_cast<double>(r[i].weight);
            if (hCos)
                hCos[i] = static_cast<double>(r[i].cosExit);
            if (hPos) {
                hPos[3 * i] = r[i].position.x;
                hPos[3 * i + 1] = r[i].position.y;
                hPos[3 * i + 2] = r[i].position.z;
            }
            if (hDir) {
                hDir[3 * i] = r[i].direction.x;
                hDir[3 * i + 1] = r[i].direction.y;
                hDir[3 * i + 2] = r[i].direction.z;
            }
        }
    }
    if (hb && (hRefl || hTrans)) {
        std::vector<T> a(hb), b(hb);
        cuda::check(cudaMemcpy(a.data(), refl.data(), sizeof(T) * hb, cudaMemcpyDeviceToHost), "D2H");
        cuda::check(cudaMemcpy(b.data(), trans.data(), sizeof(T) * hb, cudaMemcpyDeviceToHost), "D2H");
        for (std::uint32_t k = 0; k < hb; ++k) {
            if (hRefl)
                hRefl[k] = a[k];
            if (hTrans)
                hTrans[k] = b[k];
        }
    }
    if (hCounts)
        cuda::check(cudaMemcpy(hCounts, counts.data(), 40, cudaMemcpyDeviceToHost), "D2H");
    if (tr.ids != 0u) {
        std::vector<std::uint32_t> kept(tr.ids);
        cuda::check(cudaMemcpy(kept.data(), traceCounts.data(), 4u * tr.ids, cudaMemcpyDeviceToHost), "D2H");
        if (tr.hCounts)
            std::memcpy(tr.hCounts, kept.data(), 4u * tr.ids);
        if (tr.hTruncated)
            cuda::check(cudaMemcpy(tr.hTruncated, traceTruncated.data(), 4u * tr.ids, cudaMemcpyDeviceToHost), "D2H");
        if (tr.hVertices && traceSlots != 0u) {
            std::vector<TraceVertexT<T>> v(traceSlots);
            cuda::check(cudaMemcpy(v.data(), traceVertices.data(), sizeof(TraceVertexT<T>) * traceSlots,
                                   cudaMemcpyDeviceToHost),
                        "D2H");
            for (std::uint64_t id = 0; id < tr.ids; ++id)
                for (std::uint32_t j = 0; j < tr.vertices; ++j) {
                    const std::size_t k = static_cast<std::size_t>(id) * tr.vertices + j;
                    gf_trace_vertex out{};
                    if (j < kept[id]) {
                        const TraceVertexT<T>& a = v[k];
                        out.kind = static_cast<std::uint32_t>(a.kind);
                        out.scatter_count = a.scatterCount;
                        out.position[0] = a.position.x;
                        out.position[1] = a.position.y;
                        out.position[2] = a.position.z;
                        out.direction[0] = a.direction.x;
                        out.direction[1] = a.direction.y;
                        out.direction[2] = a.direction.z;
                    }
                    tr.hVertices[k] = out;
                }
        }
    }
    if (hStats) {
        std::memset(hStats, 0, sizeof(*hStats));
        hStats->completed_batches = stats.completedBatches;
        hStats->partition_batches = stats.partitionBatches;
        hStats->kernel_launches = stats.kernelLaunches;
        hStats->loop_iterations = stats.loopIterations;
        hStats->generated = exec == GF_EXEC_FLOW ? stats.sourceGenerated : n;
        hStats->sunk = exec == GF_EXEC_FLOW ? stats.sourceSunk : n;
        hStats->pool_chunks = stats.poolChunks;
        hStats->peak_live_chunks = stats.peakLiveChunks;
        hStats->peak_reserved_chunks = stats.peakReservedChunks;
        hStats->peak_ready_chunks = stats.peakReadyChunks;
        hStats->seconds = sec;
        hStats->setup_seconds = stats.setupSeconds;
        hStats->loop_seconds = stats.loopSeconds;
        hStats->partition_launches = stats.partitionLaunches;
    }
}

} // namespace

namespace {

gf_status runPhoton(uint64_t seed, uint64_t first_id, uint64_t n, const gf_photon_params* h_params, int exec,
                    uint32_t chunk_capacity, uint32_t live_particles, uint32_t batch_chunks, uint32_t* h_event,
                    uint32_t* h_scatter_count, double* h_weight, double* h_cos_exit, double* h_position,
                    double* h_direction, double* h_refl, double* h_trans, uint64_t* h_event_counts,
                    gf_flow_stats* h_stats, const TraceRequest& tr)
{
    if (h_params == nullptr || (exec != GF_EXEC_FLOW && exec != GF_EXEC_FUSED) ||
        (h_params->model != GF_PHOTON_ANALOG && h_params->model != GF_PHOTON_WEIGHTED))
        return GF_ERR_ARGUMENT;
    const gf_photon_params P = *h_params;
    if (!(P.thickness > 0.0) || P.sigma_s < 0.0 || P.sigma_a < 0.0 || P.max_scatters > 0xFFFFu ||
        (P.model == GF_PHOTON_WEIGHTED && (!(P.sigma_s + P.sigma_a > 0.0) || P.g <= -1.0 || P.g >= 1.0 ||
                                           !(P.roulette_survival > 0.0) || P.roulette_survival > 1.0)))
        return GF_ERR_ARGUMENT;
    if (n != 0u && first_id + n - 1u > 0xFFFFFFFFull)
        return GF_ERR_RANGE;
    return gf_flows_guard([&] {
        if (P.fp64)
            runTyped<double>(seed, first_id, n, P, exec, chunk_capacity, live_particles, batch_chunks, h_event,
                             h_scatter_count, h_weight, h_cos_exit, h_position, h_direction, h_refl, h_trans,
                             h_event_counts, h_stats, tr);
        else
            runTyped<float>(seed, first_id, n, P, exec, chunk_capacity, live_particles, batch_chunks, h_event,
                            h_scatter_count, h_weight, h_cos_exit, h_position, h_direction, h_refl, h_trans,
                            h_event_counts, h_stats, tr);
    });
}

} // namespace

extern "C" gf_status gf_run_photon(uint64_t seed, uint64_t first_id, uint64_t n, const gf_photon_params* h_params,
                                   int exec, uint32_t chunk_capacity, uint32_t live_particles, uint32_t batch_chunks,
                                   uint32_t* h_event, uint32_t* h_scatter_count, double* h_weight, double* h_cos_exit,
                                   double* h_position, double* h_direction, double* h_refl, double* h_trans,
                                   uint64_t* h_event_counts, gf_flow_stats* h_stats)
{
    return runPhoton(seed, first_id, n, h_params, exec, chunk_capacity, live_particles, batch_chunks, h_event,
                     h_scatter_count, h_weight, h_cos_exit, h_position, h_direction, h_refl, h_trans, h_event_counts,
                     h_stats, TraceRequest{});
}

extern "C" gf_status gf_run_photon_traced(uint64_t seed, uint64_t first_id, uint64_t n,
                                          const gf_photon_params* h_params, int exec, uint32_t chunk_capacity,
                                          uint32_t live_particles, uint32_t batch_chunks, uint32_t* h_event,
                                          uint32_t* h_scatter_count, double* h_weight, double* h_cos_exit,
                                          double* h_position, double* h_direction, double* h_refl, double* h_trans,
                                          uint64_t* h_event_counts, gf_flow_stats* h_stats, uint32_t trace_photons,
                                          uint32_t trace_vertices, gf_trace_vertex* h_trace_vertices,
                                          uint32_t* h_trace_counts, uint32_t* h_trace_truncated)
{
    TraceRequest tr;
    tr.ids = trace_photons < n ? trace_photons : n;
    tr.vertices = trace_vertices;
    tr.hVertices = h_trace_vertices;
    tr.hCounts = h_trace_counts;
    tr.hTruncated = h_trace_truncated;
    if (tr.ids != 0u && first_id != 0u)
        return GF_ERR_ARGUMENT;
    // the id-major vertex array must be addressable: ids x vertices x 56 bytes within 2^62
    if (tr.ids != 0u && trace_vertices != 0u && tr.ids > (std::uint64_t{1} << 56) / trace_vertices)
        return GF_ERR_RANGE;
    return runPhoton(seed, first_id, n, h_params, exec, chunk_capacity, live_particles, batch_chunks, h_event,
                     h_scatter_count, h_weight, h_cos_exit, h_position, h_direction, h_refl, h_trans, h_event_counts,
                     h_stats, tr);
}

// Enqueues the FP32 transport of photons [0, n) with the parameters' model on `stream`, writing one
// terminal record per photon to d_records (TerminalT<float>[n]) and counting deliveries in
// d_visits (zeroed by the caller); failures go to d_status. Used by the request server.
void gf_photon_enqueue_f32(cudaStream_t stream, const gf_photon_params& P, std::uint64_t seed, std::uint64_t n,
                           void* d_records, std::uint32_t* d_visits, std::uint32_t* d_status, std::uint32_t sms)
{
    if (n == 0u)
        return;
    const SlabT<float> slab{static_cast<float>(P.thickness), static_cast<float>(P.sigma_s),
                            static_cast<float>(P.sigma_a)};
    RecordTerminalT<float> terminal{static_cast<TerminalT<float>*>(d_records), d_visits, nullptr, nullptr, 0u, nullptr};
    const unsigned blocks = static_cast<unsigned>(std::min<std::uint64_t>((n + 255u) / 256u, sms * 64u));
    if (P.model == GF_PHOTON_ANALOG)
        transport_kernel<float><<<blocks, 256, 0, stream>>>(ProposeFlightT<float>{slab, P.max_scatters},
                                                            AdvanceToEventT<float>{slab}, ScatterT<float>{P.isotropic != 0},
                                                            terminal, gf::mix64(seed), 0u, n, d_status);
    else
        transport_kernel<float><<<blocks, 256, 0, stream>>>(
            ProposeWeightedT<float>{slab,
                                    WeightedT<float>{static_cast<float>(P.g), static_cast<float>(P.roulette_threshold),
                                                     static_cast<float>(P.roulette_survival)},
                                    P.max_scatters},
            AdvanceToEventT<float>{slab}, ScatterHGT<float>{static_cast<float>(P.g)}, terminal, gf::mix64(seed), 0u, n,
            d_status);
    cuda::check(cudaGetLastError(), "photon transport launch");
}

// Size of one FP32 terminal record (the request server sizes its buffers with it).
std::size_t gf_photon_record_bytes_f32() { return sizeof(TerminalT<float>); }
