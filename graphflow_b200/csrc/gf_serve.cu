// Request server over the hot path: a stream of whole-flow requests (particle_feedback, photon
// slab transport, two-node dense classify chains), each with its own size and seed, served either
// one at a time through the C++ Flow (the plain per-batch form) or with continuous batching: a
// request is admitted as soon as a stream slot and its device memory (from one arena capped by the
// caller) are free, its whole flow runs on the device on its own stream with no host round trip,
// and requests that arrive meanwhile are admitted while others run, so their work overlaps.
//
// Every request's result is reduced to an order-independent digest (a 64-bit sum of a mix of each
// particle's id and result), so a request's digest is the same alone, in the mix, and in either
// form. Latency = completion time - arrival time.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <thread>
#include <vector>

#include "../examples/dense_chain.cuh"
#include "../examples/particle_feedback.cuh"
#include "gf_device_chain.cuh"

gf_status gf_flows_guard(const std::function<void()>& body); // gf_flows.cu
void gf_photon_enqueue_f32(cudaStream_t stream, const gf_photon_params& P, std::uint64_t seed, std::uint64_t n,
                           void* d_records, std::uint32_t* d_visits, std::uint32_t* d_status,
                           std::uint32_t sms);        // gf_photon.cu
std::size_t gf_photon_record_bytes_f32();             // gf_photon.cu

namespace {

using namespace graphflow;

constexpr std::uint32_t kChainNodes = 2u;
constexpr std::uint32_t kFeedbackVisits = 64u;
constexpr std::uint64_t kGolden = 0x9E3779B97F4A7C15ull;

// ---- digests (host and device) ----
GF_HD std::uint64_t digest_feedback(std::uint64_t id, std::uint32_t weight, std::uint32_t capped)
{
    return gf::mix64((id * kGolden) ^ ((static_cast<std::uint64_t>(capped != 0u) << 32) | weight));
}
GF_HD std::uint64_t digest_photon(std::uint64_t id, std::uint32_t event, std::uint32_t weightBits,
                                  std::uint32_t cosBits)
{
    return gf::mix64((id * kGolden) ^ (static_cast<std::uint64_t>(event) << 56) ^
                     gf::mix64((static_cast<std::uint64_t>(weightBits) << 32) | cosBits));
}
GF_HD std::uint64_t digest_port(std::uint64_t id, std::uint32_t port)
{
    return gf::mix64((id * kGolden) ^ (static_cast<std::uint64_t>(port) << 40));
}

GF_D void add_digest(unsigned long long* acc, std::uint64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31u) == 0u)
        atomicAdd(acc, static_cast<unsigned long long>(v));
}

// All three kernels run a whole number of warps over a grid-stride loop padded to full warps.
__global__ void digest_feedback_kernel(const std::uint32_t* weights, const std::uint32_t* capped, std::uint64_t n,
                                       unsigned long long* acc)
{
    std::uint64_t sum = 0;
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        sum += digest_feedback(i, weights[i], capped[i]);
    add_digest(acc, sum);
}

struct PhotonRecordF32 { // TerminalT<float> as stored (event, scatter count, weight, cos, position, direction)
    std::uint32_t event, scatterCount;
    float weight, cosExit, x, y, z, ux, uy, uz;
};

__global__ void digest_photon_kernel(const PhotonRecordF32* rec, std::uint64_t n, unsigned long long* acc)
{
    std::uint64_t sum = 0;
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        sum += digest_photon(i, rec[i].event, __float_as_uint(rec[i].weight), __float_as_uint(rec[i].cosExit));
    add_digest(acc, sum);
}

__global__ void digest_port_kernel(const std::uint32_t* portOf, std::uint64_t n, unsigned long long* acc)
{
    std::uint64_t sum = 0;
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        sum += digest_port(i, portOf[i]);
    add_digest(acc, sum);
}

__global__ void fill_u32_kernel(std::uint32_t* p, std::uint64_t n, std::uint32_t v)
{
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    for (std::uint64_t i = static_cast<std::uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        p[i] = v;
}

// ---- the two-node dense chain: gf_device_chain.cuh with a device-resident chunk pool ----
gf::DeviceChainLayout chainLayout(std::uint64_t n, std::uint32_t bins)
{
    return gf::DeviceChainLayout(n, bins, kChainNodes, outputChunkBound(n, gf::kChainCapacity, bins));
}

void enqueueChain(cudaStream_t s, char* base, const gf::DeviceChainLayout& L, std::uint64_t seed,
                  std::uint32_t* status, unsigned long long* acc, std::uint32_t sms)
{
    gf::enqueueDeviceChain(s, base, L, GF_DIST_UNIFORM, nullptr, seed, status, sms);
    const unsigned g = static_cast<unsigned>(std::min<std::uint64_t>((std::max<std::uint64_t>(L.n, 1u) + 255u) / 256u,
                                                                     sms * 8u));
    digest_port_kernel<<<g, 256, 0, s>>>(reinterpret_cast<const std::uint32_t*>(base + L.portOf), L.n, acc);
    cuda::check(cudaGetLastError(), "chain digest launch");
}

// ---- requests ----
gf_photon_params servedPhotonParams()
{
    gf_photon_params p{};
    p.thickness = 1.0;
    p.sigma_s = 10.0;
    p.sigma_a = 0.1;
    p.g = 0.9;
    p.roulette_threshold = 1e-4;
    p.roulette_survival = 0.1;
    p.max_scatters = 0xFFFFu;
    p.hist_bins = 256u;
    p.model = GF_PHOTON_WEIGHTED;
    p.isotropic = 0;
    p.fp64 = 0;
    return p;
}

std::uint64_t footprint(const gf_request& r)
{
    auto up = [](std::uint64_t v) { return (v + 255u) & ~std::uint64_t(255u); };
    const std::uint64_t m = std::max<std::uint64_t>(r.n, 1u);
    switch (r.kind) {
    case GF_REQ_PARTICLE_FEEDBACK:
        return 2u * up(m * 4u);
    case GF_REQ_PHOTON:
        return up(m * gf_photon_record_bytes_f32()) + up(m * 4u);
    default:
        return chainLayout(r.n, r.bins).total;
    }
}

// Result slot in pinned host memory: digest, status word, particles.
struct Pinned {
    unsigned long long digest;
    std::uint32_t status;
    std::uint32_t pad;
};

// Enqueues request r fully on stream s inside its arena block; the digest and status land in the
// device words dev[0..1] and are copied to *host before the completion event.
void enqueueRequest(cudaStream_t s, const gf_request& r, char* block, unsigned long long* dev, Pinned* host,
                    std::uint32_t sms)
{
    auto* acc = dev;
    auto* status = reinterpret_cast<std::uint32_t*>(dev + 1);
    cuda::check(cudaMemsetAsync(dev, 0, 16u, s), "memset");
    const std::uint64_t m = std::max<std::uint64_t>(r.n, 1u);
    const unsigned g = static_cast<unsigned>(std::min<std::uint64_t>((m + 255u) / 256u, sms * 8u));
    if (r.kind == GF_REQ_PARTICLE_FEEDBACK) {
        auto* weights = reinterpret_cast<std::uint32_t*>(block);
        auto* capped = reinterpret_cast<std::uint32_t*>(block + ((m * 4u + 255u) & ~std::uint64_t(255u)));
        fill_u32_kernel<<<g, 256, 0, s>>>(weights, m, particle::missingWeight);
        fill_u32_kernel<<<g, 256, 0, s>>>(capped, m, 0u);
        particle::launchParticleTransport(s, r.seed, 0u, r.n, kFeedbackVisits, weights, capped, status, sms);
        digest_feedback_kernel<<<g, 256, 0, s>>>(weights, capped, r.n, acc);
    } else if (r.kind == GF_REQ_PHOTON) {
        auto* rec = block;
        auto* visits = reinterpret_cast<std::uint32_t*>(
            block + ((m * gf_photon_record_bytes_f32() + 255u) & ~std::uint64_t(255u)));
        fill_u32_kernel<<<g, 256, 0, s>>>(visits, m, 0u);
        gf_photon_enqueue_f32(s, servedPhotonParams(), r.seed, r.n, rec, visits, status, sms);
        digest_photon_kernel<<<g, 256, 0, s>>>(reinterpret_cast<const PhotonRecordF32*>(rec), r.n, acc);
    } else {
        enqueueChain(s, block, chainLayout(r.n, r.bins), r.seed, status, acc, sms);
    }
    cuda::check(cudaGetLastError(), "request launch");
    cuda::check(cudaMemcpyAsync(host, dev, 16u, cudaMemcpyDeviceToHost, s), "D2H");
}

// First-fit allocator over one device block (offsets in bytes, 256-byte granules).
class Arena {
public:
    explicit Arena(std::uint64_t bytes) : m_bytes(bytes) { m_free[0] = bytes; }
    bool alloc(std::uint64_t size, std::uint64_t& off)
    {
        size = (size + 255u) & ~std::uint64_t(255u);
        for (auto it = m_free.begin(); it != m_free.end(); ++it) {
            if (it->second >= size) {
                off = it->first;
                const std::uint64_t rest = it->second - size;
                m_free.erase(it);
                if (rest)
                    m_free[off + size] = rest;
                m_used += size;
                return true;
            }
        }
        return false;
    }
    void release(std::uint64_t off, std::uint64_t size)
    {
        size = (size + 255u) & ~std::uint64_t(255u);
        m_used -= size;
        auto it = m_free.emplace(off, size).first;
        auto next = std::next(it);
        if (next != m_free.end() && it->first + it->second == next->first) {
            it->second += next->second;
            m_free.erase(next);
        }
        if (it != m_free.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                m_free.erase(it);
            }
        }
    }
    std::uint64_t used() const { return m_used; }

private:
    std::uint64_t m_bytes;
    std::uint64_t m_used = 0;
    std::map<std::uint64_t, std::uint64_t> m_free;
};

double secondsSince(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void waitUntil(std::chrono::steady_clock::time_point t0, double when)
{
    for (;;) {
        const double now = secondsSince(t0);
        if (now >= when)
            return;
        if (when - now > 2e-3)
            std::this_thread::sleep_for(std::chrono::microseconds(500));
    }
}

// ---- plain form: one request at a time through the C++ Flow, reference runner, plain partitions ----
std::uint64_t hostDigestFeedback(const std::vector<std::uint32_t>& w, const std::vector<std::uint32_t>& c)
{
    std::uint64_t d = 0;
    for (std::size_t i = 0; i < w.size(); ++i)
        d += digest_feedback(i, w[i], c[i]);
    return d;
}

gf_status runPlain(const gf_request& r, std::uint64_t& digest)
{
    const std::uint64_t m = std::max<std::uint64_t>(r.n, 1u);
    if (r.kind == GF_REQ_PARTICLE_FEEDBACK) {
        std::vector<std::uint32_t> w(m), c(m);
        gf_flow_stats st{};
        const gf_status rc = gf_run_particle_feedback(r.seed, r.n, kFeedbackVisits, 1024u, 4096u, 8u, 0,
                                                      GF_LAYOUT_SOA, w.data(), c.data(), &st);
        w.resize(r.n);
        c.resize(r.n);
        digest = hostDigestFeedback(w, c);
        return rc;
    }
    if (r.kind == GF_REQ_PHOTON) {
        const gf_photon_params p = servedPhotonParams();
        std::vector<std::uint32_t> ev(m);
        std::vector<double> w(m), cs(m);
        gf_flow_stats st{};
        const gf_status rc = gf_run_photon(r.seed, 0u, r.n, &p, GF_EXEC_FLOW, 8192u, 0u, 8u, ev.data(), nullptr,
                                           w.data(), cs.data(), nullptr, nullptr, nullptr, nullptr, nullptr, &st);
        std::uint64_t d = 0;
        for (std::uint64_t i = 0; i < r.n; ++i) {
            const float wf = static_cast<float>(w[i]), cf = static_cast<float>(cs[i]);
            std::uint32_t wb, cb;
            std::memcpy(&wb, &wf, 4);
            std::memcpy(&cb, &cf, 4);
            d += digest_photon(i, ev[i], wb, cb);
        }
        digest = d;
        return rc;
    }
    std::vector<std::uint32_t> port(m);
    gf_flow_stats st{};
    const gf_status rc = gf_run_dense_chain(r.seed, r.n, r.bins, kChainNodes, GF_DIST_UNIFORM, 1.0, gf::kChainCapacity,
                                            16384u, 8u, 0, GF_LAYOUT_SOA, port.data(), &st);
    std::uint64_t d = 0;
    for (std::uint64_t i = 0; i < r.n; ++i)
        d += digest_port(i, port[i]);
    digest = d;
    return rc;
}

} // namespace

bool gf_runner_batched();  // gf_capi.cu
bool gf_device_resident(); // gf_capi.cu

extern "C" gf_status gf_serve(const gf_request* h_requests, uint32_t n_requests, int mode, uint64_t memory_cap_bytes,
                              uint32_t max_inflight, gf_request_result* h_results, gf_serve_stats* h_stats)
{
    if ((n_requests != 0u && (h_requests == nullptr || h_results == nullptr)) ||
        (mode != GF_SERVE_PLAIN && mode != GF_SERVE_BATCHED && mode != GF_SERVE_FLOW_DEVICE) || max_inflight == 0u ||
        max_inflight > 256u)
        return GF_ERR_ARGUMENT;
    for (uint32_t i = 0; i < n_requests; ++i) {
        const gf_request& r = h_requests[i];
        if (r.kind > GF_REQ_DENSE_CHAIN || (r.kind == GF_REQ_DENSE_CHAIN && r.bins != 2u && r.bins != 8u &&
                                             r.bins != 32u) ||
            r.n > 0xFFFFFFFFull || (i != 0u && r.arrival_s < h_requests[i - 1u].arrival_s))
            return GF_ERR_ARGUMENT;
    }
    return gf_flows_guard([&] {
        cuda::Device device = cuda::Device::current();
        device.makeCurrent();
        const std::uint32_t sms = device.multiProcessorCount();
        if (gf_photon_record_bytes_f32() != sizeof(PhotonRecordF32))
            throw std::logic_error("gf_serve: photon record layout mismatch");
        if (n_requests != 0u)
            std::memset(h_results, 0, sizeof(gf_request_result) * n_requests);
        gf_serve_stats stats{};
        if (mode == GF_SERVE_PLAIN || mode == GF_SERVE_FLOW_DEVICE) {
            // one request at a time through the Flow: the reference runner (one-chunk sinks, one
            // dispatch per iteration), or the same graphs run device-resident
            const int saved = gf_runner_batched() ? 1 : 0, savedDevice = gf_device_resident() ? 1 : 0;
            auto restore = [&] {
                gf_set_tuning("runner_batched", saved);
                gf_set_tuning("device_resident", savedDevice);
            };
            if (mode == GF_SERVE_PLAIN) {
                gf_set_tuning("runner_batched", 0);
                gf_set_tuning("device_resident", 0);
            } else {
                gf_set_tuning("device_resident", 1);
            }
            try {
                const auto t0 = std::chrono::steady_clock::now();
                for (uint32_t i = 0; i < n_requests; ++i) {
                    waitUntil(t0, h_requests[i].arrival_s);
                    h_results[i].admit_s = secondsSince(t0);
                    std::uint64_t d = 0;
                    h_results[i].status = static_cast<uint32_t>(runPlain(h_requests[i], d));
                    h_results[i].digest = d;
                    h_results[i].done_s = secondsSince(t0);
                }
                stats.seconds = secondsSince(t0);
                stats.peak_inflight = n_requests ? 1u : 0u;
            } catch (...) {
                restore();
                throw;
            }
            restore();
            if (h_stats)
                *h_stats = stats;
            return;
        }
        // continuous batching
        std::uint64_t need = 0;
        for (uint32_t i = 0; i < n_requests; ++i)
            need = std::max(need, footprint(h_requests[i]));
        const std::uint64_t arenaBytes = std::min<std::uint64_t>(memory_cap_bytes, std::max<std::uint64_t>(need, 1u) *
                                                                                       max_inflight);
        cuda::Buffer<char> arena(std::max<std::uint64_t>(arenaBytes, 256u));
        cuda::Buffer<unsigned long long> words(2u * max_inflight);
        cuda::HostBuffer<Pinned> pinned(max_inflight);
        std::vector<cudaStream_t> streams(max_inflight);
        std::vector<cudaEvent_t> events(max_inflight);
        for (uint32_t k = 0; k < max_inflight; ++k) {
            cuda::check(cudaStreamCreateWithFlags(&streams[k], cudaStreamNonBlocking), "stream");
            cuda::check(cudaEventCreateWithFlags(&events[k], cudaEventDisableTiming), "event");
        }
        struct Slot {
            bool busy = false;
            uint32_t req = 0;
            std::uint64_t off = 0, size = 0;
        };
        std::vector<Slot> slots(max_inflight);
        Arena alloc(arenaBytes);
        std::deque<uint32_t> pending;
        uint32_t next = 0, done = 0, inflight = 0;
        const auto t0 = std::chrono::steady_clock::now();
        try {
            while (done < n_requests) {
                bool progress = false;
                const double now = secondsSince(t0);
                while (next < n_requests && h_requests[next].arrival_s <= now)
                    pending.push_back(next++);
                for (uint32_t k = 0; k < max_inflight; ++k) {
                    Slot& sl = slots[k];
                    if (!sl.busy)
                        continue;
                    const cudaError_t q = cudaEventQuery(events[k]);
                    if (q == cudaErrorNotReady)
                        continue;
                    cuda::check(q, "event");
                    gf_request_result& res = h_results[sl.req];
                    res.digest = pinned[k].digest;
                    res.status = pinned[k].status;
                    res.done_s = secondsSince(t0);
                    alloc.release(sl.off, sl.size);
                    sl.busy = false;
                    --inflight;
                    ++done;
                    progress = true;
                }
                while (!pending.empty()) {
                    const uint32_t ri = pending.front();
                    const gf_request& r = h_requests[ri];
                    const std::uint64_t fp = footprint(r);
                    if (fp > arenaBytes) { // can never fit under the cap
                        h_results[ri].status = GF_ERR_RANGE;
                        h_results[ri].admit_s = h_results[ri].done_s = secondsSince(t0);
                        pending.pop_front();
                        ++done;
                        progress = true;
                        continue;
                    }
                    uint32_t k = 0;
                    while (k < max_inflight && slots[k].busy)
                        ++k;
                    std::uint64_t off = 0;
                    if (k == max_inflight || !alloc.alloc(fp, off))
                        break; // head of line waits for a slot or memory
                    Slot& sl = slots[k];
                    sl = Slot{true, ri, off, fp};
                    h_results[ri].admit_s = secondsSince(t0);
                    enqueueRequest(streams[k], r, arena.data() + off, words.data() + 2u * k, &pinned[k], sms);
                    cuda::check(cudaEventRecord(events[k], streams[k]), "event record");
                    ++inflight;
                    stats.peak_inflight = std::max(stats.peak_inflight, inflight);
                    stats.peak_bytes = std::max<std::uint64_t>(stats.peak_bytes, alloc.used());
                    pending.pop_front();
                    progress = true;
                }
                if (!progress) {
                    if (inflight == 0u && next < n_requests)
                        waitUntil(t0, h_requests[next].arrival_s);
                    else
                        std::this_thread::yield();
                }
            }
            stats.seconds = secondsSince(t0);
        } catch (...) {
            cudaDeviceSynchronize();
            for (uint32_t k = 0; k < max_inflight; ++k) {
                cudaStreamDestroy(streams[k]);
                cudaEventDestroy(events[k]);
            }
            throw;
        }
        for (uint32_t k = 0; k < max_inflight; ++k) {
            cudaStreamDestroy(streams[k]);
            cudaEventDestroy(events[k]);
        }
        if (h_stats)
            *h_stats = stats;
    });
}
