// Device-side vocabulary of the C++ front end: the CUDA device type, the status word, update
// results, keyed RNG engines with per-payload stream fields, and the functor calling rules.
//
// Reference (paths inside graphFlow's include/graphFlow): flow/Status.hpp:21-96,
// flow/Concepts.hpp:126-200 (functor shapes: optional accelerator, then optional engine, then
// optional status, then the payload), rng/ParticleRng.hpp:35-170 (stream key, stream traits).
#pragma once

#include <cstdint>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include <cuda_runtime.h>

#include "core.hpp"
#include "gf_device.cuh"
#include "policy.hpp"

namespace graphflow {

// ---- status word (flow/Status.hpp:21-96) ----
enum class StatusCode : std::uint32_t { ok = 0u, invalid = 1u, overflow = 2u };

__host__ __device__ inline StatusCode decodeStatus(std::uint32_t w)
{
    return w == 0u ? StatusCode::ok : (w == 2u ? StatusCode::overflow : StatusCode::invalid);
}

inline const char* statusCodeName(StatusCode c)
{
    return c == StatusCode::ok ? "ok" : (c == StatusCode::overflow ? "overflow" : "invalid");
}

class Status {
public:
    Status() = default;
    __device__ explicit Status(std::uint32_t* word) : m_word(word) {}
    __device__ void set(StatusCode code) const
    {
        if (m_word != nullptr)
            atomicCAS(m_word, 0u, static_cast<std::uint32_t>(code));
    }
    __device__ void fail(StatusCode code) const { set(code); }
    __device__ StatusCode code() const { return m_word == nullptr ? StatusCode::ok : decodeStatus(*m_word); }
    __device__ bool ok() const { return code() == StatusCode::ok; }

private:
    std::uint32_t* m_word = nullptr;
};

// ---- updater result (flow/Concepts.hpp) ----
enum class UpdateResult : std::uint32_t { success = 0u, overflow = 1u, invalid = 2u };

// No-op updater (the default of Flow::partition).
struct NoUpdate {
    template <typename TBin, typename TPayload>
    __device__ UpdateResult operator()(TBin, TPayload&) const
    {
        return UpdateResult::success;
    }
};

// ---- accelerator token: functors may take a leading `auto const& acc` argument ----
struct Acc {
    __device__ std::uint32_t threadIndex() const { return blockIdx.x * blockDim.x + threadIdx.x; }
};

namespace rng {

using Engine = gf::Engine;

inline constexpr std::uint64_t maxStreamId = 0xFFFFFFFFull;
inline constexpr std::uint64_t maxStreamEvent = 0xFFFFull;
inline constexpr std::uint32_t maxStreamPurpose = 0xFFFFu;

// rng/ParticleRng.hpp:51-54: node key k owns purposes 2k (functor) and 2k+1 (updater).
constexpr std::uint32_t streamPurposeForNode(std::uint64_t nodeKey, std::uint32_t sub = 0u)
{
    return static_cast<std::uint32_t>((nodeKey << 1u) | (sub & 1u));
}

// rng/ParticleRng.hpp:131-157: default stream fields read `id` and `visit` or `scatterCount`.
template <typename TPayload>
struct StreamTraits {
    __host__ __device__ static std::uint64_t id(const TPayload& p)
    {
        if constexpr (requires { p.id; })
            return static_cast<std::uint64_t>(p.id);
        else
            return 0u;
    }
    __host__ __device__ static std::uint64_t event(const TPayload& p)
    {
        if constexpr (requires { p.visit; })
            return static_cast<std::uint64_t>(p.visit);
        else if constexpr (requires { p.scatterCount; })
            return static_cast<std::uint64_t>(p.scatterCount);
        else
            return 0u;
    }
};

__device__ inline Engine makeEngine(std::uint64_t seedMixed, std::uint64_t id, std::uint64_t event,
                                    std::uint32_t purpose)
{
    return Engine(gf::stream_key(seedMixed, id, event, purpose));
}

template <typename TPayload>
__device__ inline Engine engineFor(std::uint64_t seedMixed, const TPayload& p, std::uint32_t purpose)
{
    return makeEngine(seedMixed, StreamTraits<TPayload>::id(p), StreamTraits<TPayload>::event(p), purpose);
}

// Word-to-real conversion of this library (one 32-bit draw per real), [0, 1).
template <typename T>
__device__ inline T uniform(Engine& e)
{
    if constexpr (std::is_same_v<T, float>)
        return gf::uniform_f32(e());
    else
        return static_cast<T>(gf::uniform_f64(e()));
}

} // namespace rng

// ---- functor calling rules (flow/Concepts.hpp:126-200, flow/Execution.hpp:88-110) ----
template <typename F, typename... A>
__device__ inline decltype(auto) invokeWithContext(const F& f, rng::Engine& engine, Status& status, A&&... args)
{
    const Acc acc{};
    if constexpr (std::is_invocable_v<const F&, const Acc&, rng::Engine&, Status&, A...>)
        return f(acc, engine, status, std::forward<A>(args)...);
    else if constexpr (std::is_invocable_v<const F&, const Acc&, rng::Engine&, A...>)
        return f(acc, engine, std::forward<A>(args)...);
    else if constexpr (std::is_invocable_v<const F&, const Acc&, Status&, A...>)
        return f(acc, status, std::forward<A>(args)...);
    else if constexpr (std::is_invocable_v<const F&, const Acc&, A...>)
        return f(acc, std::forward<A>(args)...);
    else if constexpr (std::is_invocable_v<const F&, rng::Engine&, Status&, A...>)
        return f(engine, status, std::forward<A>(args)...);
    else if constexpr (std::is_invocable_v<const F&, rng::Engine&, A...>)
        return f(engine, std::forward<A>(args)...);
    else if constexpr (std::is_invocable_v<const F&, Status&, A...>)
        return f(status, std::forward<A>(args)...);
    else
        return f(std::forward<A>(args)...);
}

// Result type of a functor under the calling rules above, from its declared signature. Host and
// device compilation must agree on it (it selects kernel instantiations), so it is computed with
// std::invoke_result on the functor itself, never through a deduced `decltype(auto)` body.
// Classifiers therefore declare their return type explicitly (as the reference's functors do).
template <typename F, typename... A>
constexpr auto contextResultTag()
{
    if constexpr (std::is_invocable_v<const F&, const Acc&, rng::Engine&, Status&, A...>)
        return std::type_identity<std::invoke_result_t<const F&, const Acc&, rng::Engine&, Status&, A...>>{};
    else if constexpr (std::is_invocable_v<const F&, const Acc&, rng::Engine&, A...>)
        return std::type_identity<std::invoke_result_t<const F&, const Acc&, rng::Engine&, A...>>{};
    else if constexpr (std::is_invocable_v<const F&, const Acc&, Status&, A...>)
        return std::type_identity<std::invoke_result_t<const F&, const Acc&, Status&, A...>>{};
    else if constexpr (std::is_invocable_v<const F&, const Acc&, A...>)
        return std::type_identity<std::invoke_result_t<const F&, const Acc&, A...>>{};
    else if constexpr (std::is_invocable_v<const F&, rng::Engine&, Status&, A...>)
        return std::type_identity<std::invoke_result_t<const F&, rng::Engine&, Status&, A...>>{};
    else if constexpr (std::is_invocable_v<const F&, rng::Engine&, A...>)
        return std::type_identity<std::invoke_result_t<const F&, rng::Engine&, A...>>{};
    else if constexpr (std::is_invocable_v<const F&, Status&, A...>)
        return std::type_identity<std::invoke_result_t<const F&, Status&, A...>>{};
    else
        return std::type_identity<std::invoke_result_t<const F&, A...>>{};
}

template <typename F, typename... A>
using ContextResult = typename decltype(contextResultTag<F, A...>())::type;

// Bin type of a classifier for a payload (flow/Concepts.hpp ClassifierBin).
template <typename TClassifier, typename TPayload>
using ClassifierBin = std::decay_t<ContextResult<TClassifier, const TPayload&>>;

// A transform may mutate its payload in place or return a replacement
// (flow/Execution.hpp:126-140 finishTransform).
template <typename F, typename P>
__device__ inline void applyTransform(const F& f, rng::Engine& engine, Status& status, P& p)
{
    using R = decltype(invokeWithContext(f, engine, status, p));
    if constexpr (std::is_void_v<R>)
        invokeWithContext(f, engine, status, p);
    else
        p = invokeWithContext(f, engine, status, p);
}

template <typename R>
__device__ inline std::uint32_t updateCode(R r)
{
    if constexpr (std::is_void_v<R>)
        return 0u;
    else
        return static_cast<std::uint32_t>(r);
}

namespace cuda {

// The CUDA device type of the front end (replaces alpaka's device + queue + event).
class Device {
public:
    explicit Device(int ordinal = 0) : m_ordinal(ordinal)
    {
        cudaDeviceProp p{};
        if (cudaGetDeviceProperties(&p, ordinal) != cudaSuccess)
            throw CudaError("graphflow::cuda::Device: no CUDA device " + std::to_string(ordinal));
        m_sms = static_cast<std::uint32_t>(p.multiProcessorCount);
        m_smemPerBlock = static_cast<std::uint32_t>(p.sharedMemPerBlockOptin);
        m_props.multiProcessorCount = m_sms;
        m_props.warpSize = static_cast<std::uint32_t>(p.warpSize);
        m_props.maxThreadsPerBlock = static_cast<std::uint32_t>(p.maxThreadsPerBlock);
        m_props.maxBlocksPerGrid = static_cast<std::uint32_t>(p.maxGridSize[0]);
        m_props.sharedMemPerBlockBytes = static_cast<std::uint32_t>(p.sharedMemPerBlock);
        m_props.globalMemBytes = static_cast<std::uint64_t>(p.totalGlobalMem);
    }
    // The calling thread's current device (cudaSetDevice), as the C entry points use it.
    static Device current()
    {
        int ordinal = 0;
        if (cudaGetDevice(&ordinal) != cudaSuccess)
            throw CudaError("graphflow::cuda::Device: no current CUDA device");
        return Device(ordinal);
    }
    int ordinal() const { return m_ordinal; }
    std::uint32_t multiProcessorCount() const { return m_sms; }
    std::uint32_t sharedMemPerBlock() const { return m_smemPerBlock; }
    // The fields the device policy reads (alpaka's getDeviceProperties).
    const DeviceProperties& getDeviceProperties() const { return m_props; }
    void makeCurrent() const { cudaSetDevice(m_ordinal); }

private:
    int m_ordinal;
    std::uint32_t m_sms = 0u, m_smemPerBlock = 0u;
    DeviceProperties m_props{};
};

inline void check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        cudaGetLastError(); // a reported failure does not linger as the thread's last error
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

namespace detail {
// Blocks of the front end's buffers kept for reuse, keyed by (device, exact size): a Flow run
// allocates the same storage and stage buffers as the previous run of its configuration, and
// cudaMalloc / cudaMallocHost (which pin, map and sometimes wait on the driver) cost up to
// hundreds of milliseconds where reuse costs nothing. A released block keeps the semantics of
// cudaFree: the device is synchronised first, so no queued work can still use it when it is
// handed out again. Blocks beyond the cap are freed; cached blocks are held until process exit.
class BlockCache {
public:
    BlockCache(bool host, std::size_t cap) : m_host(host), m_cap(cap) {}
    void* take(std::size_t bytes, int dev)
    {
        std::lock_guard<std::mutex> lock(m_mutex);
        auto range = m_blocks.equal_range(bytes);
        for (auto it = range.first; it != range.second; ++it)
            if (it->second.first == dev) {
                void* p = it->second.second;
                m_blocks.erase(it);
                m_cached -= bytes;
                return p;
            }
        return nullptr;
    }
    void give(void* p, std::size_t bytes, int dev)
    {
        cudaDeviceSynchronize();
        {
            std::lock_guard<std::mutex> lock(m_mutex);
            if (m_cached + bytes <= m_cap) {
                m_blocks.emplace(bytes, std::make_pair(dev, p));
                m_cached += bytes;
                return;
            }
        }
        if (m_host)
            cudaFreeHost(p);
        else
            cudaFree(p);
    }

private:
    bool m_host;
    std::size_t m_cap, m_cached = 0;
    std::mutex m_mutex;
    std::multimap<std::size_t, std::pair<int, void*>> m_blocks;
};
inline BlockCache& deviceBlocks()
{
    static BlockCache* c = new BlockCache(false, std::size_t(2) << 30); // never destroyed: no CUDA calls at exit
    return *c;
}
inline BlockCache& hostBlocks()
{
    static BlockCache* c = new BlockCache(true, std::size_t(256) << 20);
    return *c;
}
inline int currentDevice()
{
    int d = 0;
    cudaGetDevice(&d);
    return d;
}
} // namespace detail

// Owning device buffer (blocks reused through detail::deviceBlocks).
template <typename T>
class Buffer {
public:
    Buffer() = default;
    explicit Buffer(std::size_t n) : m_n(n)
    {
        if (n != 0u) {
            m_dev = detail::currentDevice();
            m_p = static_cast<T*>(detail::deviceBlocks().take(n * sizeof(T), m_dev));
            if (m_p == nullptr)
                check(cudaMalloc(&m_p, n * sizeof(T)), "cudaMalloc");
        }
    }
    Buffer(const Buffer&) = delete;
    Buffer& operator=(const Buffer&) = delete;
    Buffer(Buffer&& o) noexcept : m_p(o.m_p), m_n(o.m_n), m_dev(o.m_dev) { o.m_p = nullptr, o.m_n = 0; }
    Buffer& operator=(Buffer&& o) noexcept
    {
        if (this != &o) {
            reset();
            m_p = o.m_p;
            m_n = o.m_n;
            m_dev = o.m_dev;
            o.m_p = nullptr;
            o.m_n = 0;
        }
        return *this;
    }
    ~Buffer() { reset(); }
    T* data() const { return m_p; }
    std::size_t size() const { return m_n; }

private:
    void reset()
    {
        if (m_p != nullptr)
            detail::deviceBlocks().give(m_p, m_n * sizeof(T), m_dev);
        m_p = nullptr;
    }
    T* m_p = nullptr;
    std::size_t m_n = 0;
    int m_dev = 0;
};

// Owning pinned host buffer (the mapped staging of the reference's stages).
template <typename T>
class HostBuffer {
public:
    HostBuffer() = default;
    explicit HostBuffer(std::size_t n) : m_n(n)
    {
        if (n != 0u) {
            m_p = static_cast<T*>(detail::hostBlocks().take(n * sizeof(T), -1));
            if (m_p == nullptr)
                check(cudaMallocHost(&m_p, n * sizeof(T)), "cudaMallocHost");
        }
    }
    HostBuffer(const HostBuffer&) = delete;
    HostBuffer& operator=(const HostBuffer&) = delete;
    HostBuffer(HostBuffer&& o) noexcept : m_p(o.m_p), m_n(o.m_n) { o.m_p = nullptr, o.m_n = 0; }
    HostBuffer& operator=(HostBuffer&& o) noexcept
    {
        if (this != &o) {
            if (m_p != nullptr)
                detail::hostBlocks().give(m_p, m_n * sizeof(T), -1);
            m_p = o.m_p;
            m_n = o.m_n;
            o.m_p = nullptr;
            o.m_n = 0;
        }
        return *this;
    }
    ~HostBuffer()
    {
        if (m_p != nullptr)
            detail::hostBlocks().give(m_p, m_n * sizeof(T), -1);
    }
    T* data() const { return m_p; }
    T& operator[](std::size_t i) const { return m_p[i]; }
    std::size_t size() const { return m_n; }

private:
    T* m_p = nullptr;
    std::size_t m_n = 0;
};

// Device address of pinned host memory (cudaMallocHost memory is mapped; under unified addressing
// the address is the host pointer itself).
template <typename T>
T* mappedDevicePointer(T* host)
{
    void* d = nullptr;
    check(cudaHostGetDevicePointer(&d, host, 0), "cudaHostGetDevicePointer");
    return static_cast<T*>(d);
}

} // namespace cuda
} // namespace graphflow
