// C ABI of the device-resident chunk pool (gf_device_pool.cuh) and of the dense chain run entirely
// on the device with it (gf_device_chain.cuh).
#include <chrono>
#include <functional>
#include <string>
#include <vector>

#include "gf_device_chain.cuh"

gf_status gf_flows_guard(const std::function<void()>& body); // gf_flows.cu
bool gf_device_coop();                                        // gf_capi.cu
void gf_set_last_error(const char* message);                 // gf_flows.cu

namespace {

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

gf_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess)
        return GF_OK;
    gf_set_last_error(cudaGetErrorString(e));
    return GF_ERR_CUDA;
}

std::uint32_t current_sms()
{
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        return 1u;
    return static_cast<std::uint32_t>(n);
}

bool aligned(const void* p, std::uintptr_t a) { return (reinterpret_cast<std::uintptr_t>(p) & (a - 1u)) == 0u; }

} // namespace

extern "C" {

gf_status gf_device_pool_bytes(uint32_t num_chunks, uint64_t* h_bytes)
{
    if (h_bytes == nullptr)
        return GF_ERR_ARGUMENT;
    *h_bytes = gf::device_pool_bytes(num_chunks);
    return GF_OK;
}

gf_status gf_device_pool_init(void* stream, void* d_pool, uint32_t num_chunks)
{
    if (d_pool == nullptr || !aligned(d_pool, 16u))
        return GF_ERR_ARGUMENT;
    const unsigned g = num_chunks / gf::kPoolThreads + 1u;
    gf::pool_init_kernel<<<g < 1024u ? g : 1024u, gf::kPoolThreads, 0, as_stream(stream)>>>(
        static_cast<gf::DevicePoolHdr*>(d_pool), num_chunks);
    return cuda_status(cudaGetLastError());
}

gf_status gf_device_pool_acquire(void* stream, void* d_pool, uint32_t k, uint32_t* d_ids, uint32_t* d_status)
{
    if (d_pool == nullptr || !aligned(d_pool, 16u) || (k != 0u && d_ids == nullptr))
        return GF_ERR_ARGUMENT;
    gf::pool_acquire_kernel<<<1, gf::kPoolThreads, 0, as_stream(stream)>>>(static_cast<gf::DevicePoolHdr*>(d_pool), k,
                                                                          d_ids, d_status);
    return cuda_status(cudaGetLastError());
}

gf_status gf_device_pool_settle(void* stream, void* d_pool, const uint32_t* d_reserved, uint32_t reserved_n,
                                const uint32_t* d_used, uint32_t used, const uint32_t* d_in, uint32_t in_stride,
                                const uint32_t* d_in_count, uint32_t in_count, uint32_t* d_status)
{
    if (d_pool == nullptr || !aligned(d_pool, 16u) || (reserved_n != 0u && d_reserved == nullptr) ||
        in_stride == 0u || (d_in == nullptr && (d_in_count != nullptr || in_count != 0u)))
        return GF_ERR_ARGUMENT;
    gf::pool_settle_kernel<<<1, gf::kPoolThreads, 0, as_stream(stream)>>>(
        static_cast<gf::DevicePoolHdr*>(d_pool), d_reserved, reserved_n, d_used, used, d_in, in_stride, d_in_count,
        in_count, d_status);
    return cuda_status(cudaGetLastError());
}

gf_status gf_device_pool_read(void* stream, const void* d_pool, gf_device_pool_stats* h_stats)
{
    if (d_pool == nullptr || h_stats == nullptr)
        return GF_ERR_ARGUMENT;
    gf::DevicePoolHdr h{};
    cudaError_t e = cudaMemcpyAsync(&h, d_pool, sizeof(h), cudaMemcpyDeviceToHost, as_stream(stream));
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(as_stream(stream));
    if (e != cudaSuccess)
        return cuda_status(e);
    h_stats->num_chunks = h.num_chunks;
    h_stats->free_chunks = h.num_chunks - h.base;
    h_stats->peak_live = h.peak_live;
    h_stats->status = h.status;
    h_stats->acquired = h.acquired;
    h_stats->released = h.released;
    return GF_OK;
}

gf_status gf_run_dense_chain_device(uint64_t seed, uint64_t n, uint32_t bins, uint32_t nodes, int dist,
                                    double zipf_s, uint32_t* h_port_of, uint32_t* h_node_totals,
                                    gf_device_pool_stats* h_pool, gf_flow_stats* h_stats)
{
    if ((bins != 2u && bins != 8u && bins != 32u && bins != 64u) || nodes == 0u ||
        nodes > graphflow::dense::kMaxNodes || dist < GF_DIST_UNIFORM || dist > GF_DIST_ROUND_ROBIN ||
        (dist == GF_DIST_ZIPF && !(zipf_s > 0.0)))
        return GF_ERR_ARGUMENT;
    return gf_flows_guard([&] {
        using namespace graphflow;
        if (n != 0u && n - 1u > 0xFFFFFFFFull)
            throw std::overflow_error("graphflow::dense: particle ids are 32-bit");
        const auto t0 = std::chrono::steady_clock::now();
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::uint64_t bound = outputChunkBound(n, gf::kChainCapacity, bins);
        const std::uint32_t sms = current_sms();
        const gf::DeviceChainLayout L(n, bins, nodes, bound, gf_device_coop() ? sms * 16u : 0u);
        if (L.slots > 0xFFFFFFFFull)
            throw std::overflow_error("graphflow::dense: the device chain's pool exceeds 2^32 slots");
        cuda::Buffer<unsigned char> block(L.total);
        cuda::Buffer<double> cdf(bins);
        cuda::Buffer<std::uint32_t> status(1);
        if (dist == GF_DIST_ZIPF) {
            std::vector<double> h(bins);
            if (gf_zipf_cdf(zipf_s, bins, h.data()) != GF_OK)
                throw std::invalid_argument("graphflow::dense: Zipf exponent");
            cuda::check(cudaMemcpy(cdf.data(), h.data(), bins * sizeof(double), cudaMemcpyHostToDevice), "H2D");
        }
        cuda::check(cudaMemset(status.data(), 0, 4u), "memset");
        cudaStream_t s = nullptr;
        cuda::check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        char* base = reinterpret_cast<char*>(block.data());
        cudaEvent_t ev[2] = {nullptr, nullptr};
        cuda::check(cudaEventCreate(&ev[0]), "event");
        cuda::check(cudaEventCreate(&ev[1]), "event");
        const auto t1 = std::chrono::steady_clock::now();
        std::uint32_t launches = 0;
        float gpu_ms = 0.0f;
        cudaError_t e = cudaEventRecord(ev[0], s);
        try {
            launches = gf::enqueueDeviceChain(s, base, L, dist, dist == GF_DIST_ZIPF ? cdf.data() : nullptr, seed,
                                              status.data(), sms);
        } catch (...) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
            cudaEventDestroy(ev[0]);
            cudaEventDestroy(ev[1]);
            throw;
        }
        if (e == cudaSuccess)
            e = cudaEventRecord(ev[1], s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&gpu_ms, ev[0], ev[1]);
        cudaStreamDestroy(s);
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        cuda::check(e, "device chain");
        std::uint32_t st = 0;
        unsigned long long sunk = 0;
        gf::DevicePoolHdr pool{};
        cuda::check(cudaMemcpy(&st, status.data(), 4u, cudaMemcpyDeviceToHost), "D2H");
        cuda::check(cudaMemcpy(&sunk, base + L.sunk, 8u, cudaMemcpyDeviceToHost), "D2H");
        cuda::check(cudaMemcpy(&pool, base + L.pool, sizeof(pool), cudaMemcpyDeviceToHost), "D2H");
        if (h_port_of != nullptr && n != 0u)
            cuda::check(cudaMemcpy(h_port_of, base + L.portOf, n * 4u, cudaMemcpyDeviceToHost), "D2H");
        if (h_node_totals != nullptr)
            cuda::check(cudaMemcpy(h_node_totals, base + L.totals, static_cast<std::size_t>(nodes) * bins * 4u,
                                   cudaMemcpyDeviceToHost),
                        "D2H");
        if (h_pool != nullptr) {
            h_pool->num_chunks = pool.num_chunks;
            h_pool->free_chunks = pool.num_chunks - pool.base;
            h_pool->peak_live = pool.peak_live;
            h_pool->status = pool.status;
            h_pool->acquired = pool.acquired;
            h_pool->released = pool.released;
        }
        if (h_stats != nullptr) {
            *h_stats = gf_flow_stats{};
            h_stats->completed_batches = nodes + 2u;
            h_stats->partition_batches = nodes;
            h_stats->kernel_launches = launches;
            h_stats->generated = n;
            h_stats->sunk = sunk;
            h_stats->pool_chunks = pool.num_chunks;
            h_stats->peak_live_chunks = pool.peak_live;
            h_stats->peak_reserved_chunks = static_cast<std::uint32_t>(bound);
            h_stats->partition_launches = nodes;
            const auto t3 = std::chrono::steady_clock::now();
            h_stats->seconds = std::chrono::duration<double>(t3 - t0).count();
            h_stats->setup_seconds = std::chrono::duration<double>(t1 - t0).count();
            h_stats->loop_seconds = gpu_ms * 1e-3; // on the device, first launch to last
        }
        auto fail = [](std::uint32_t code, const std::string& what) {
            if (code == GF_ERR_TIMEOUT)
                throw SchedulerStallError(what + ": a bounded device wait ran out");
            throw BatchError(what + (code == GF_OVERFLOW ? ": overflow" : ": invalid input"));
        };
        if (st != GF_OK)
            fail(st, "graphflow::dense: the device chain failed");
        if (pool.status != GF_OK)
            fail(pool.status, "graphflow::dense: the device chain's chunk pool recorded a failure");
    });
}

} // extern "C"
