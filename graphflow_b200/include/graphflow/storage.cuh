// Payload storage of the C++ front end: fixed-layout pools of `numChunks` chunks of
// `chunkCapacity` slots, slot = chunk * capacity + offset (flow/PayloadStorage.hpp:320-880 SoA,
// core/PayloadSlotStorage.hpp AoS). Both expose a trivially copyable device view with
// load(slot) / store(slot, payload), which is what every kernel takes.
#pragma once

#include <array>
#include <cstdint>
#include <type_traits>

#include "device.cuh"

namespace graphflow {

// Field list of an SoA payload. Specialise with
//   static constexpr std::size_t count = N;
//   template <class P, class F> __host__ __device__ static void forEach(P& p, F&& f)
//   { f(p.a); f(p.b); ... }
// Each visited field becomes one device column.
template <typename T>
struct SoAFields;

namespace detail {
template <typename T>
struct FieldSizes {
    std::array<std::size_t, SoAFields<T>::count> bytes{};
    std::size_t total = 0;
    FieldSizes()
    {
        T probe{};
        std::size_t i = 0;
        SoAFields<T>::forEach(probe, [&](auto& field) {
            bytes[i++] = sizeof(field);
            total += sizeof(field);
        });
    }
};
} // namespace detail

template <typename T, typename TDevice = cuda::Device>
class SoAStorage {
    static_assert(std::is_trivially_copyable_v<T>, "graphflow::SoAStorage: payload must be trivially copyable");

public:
    using Payload = T;
    static constexpr std::size_t kFields = SoAFields<T>::count;

    struct View {
        using Payload = T;
        std::array<unsigned char*, kFields> cols;
        __device__ T load(std::uint64_t slot) const
        {
            T p{};
            std::size_t i = 0;
            SoAFields<T>::forEach(p, [&](auto& field) {
                using F = std::remove_reference_t<decltype(field)>;
                field = reinterpret_cast<const F*>(cols[i++])[slot];
            });
            return p;
        }
        __device__ void store(std::uint64_t slot, const T& p) const
        {
            std::size_t i = 0;
            T q = p;
            SoAFields<T>::forEach(q, [&](auto& field) {
                using F = std::remove_reference_t<decltype(field)>;
                reinterpret_cast<F*>(cols[i++])[slot] = field;
            });
        }
    };

    SoAStorage(const TDevice&, std::uint32_t numChunks, std::uint32_t capacity) : m_ledger(numChunks, capacity)
    {
        const detail::FieldSizes<T> sizes;
        const std::size_t slots = static_cast<std::size_t>(numChunks) * capacity;
        for (std::size_t i = 0; i < kFields; ++i) {
            m_cols[i] = cuda::Buffer<unsigned char>(slots * sizes.bytes[i]);
            m_view.cols[i] = m_cols[i].data();
        }
        m_slotBytes = sizes.total;
    }

    static std::uint64_t slotBytes()
    {
        static const detail::FieldSizes<T> sizes;
        return sizes.total;
    }
    View view() const { return m_view; }
    ChunkLedger& ledger() { return m_ledger; }
    const ChunkLedger& ledger() const { return m_ledger; }
    std::uint32_t numChunks() const { return m_ledger.numChunks(); }
    std::uint32_t chunkCapacity() const { return m_ledger.chunkCapacity(); }
    std::uint64_t slotCount() const { return static_cast<std::uint64_t>(numChunks()) * chunkCapacity(); }
    std::uint64_t base(ChunkHandle h) const { return m_ledger.base(h); }

private:
    ChunkLedger m_ledger;
    std::array<cuda::Buffer<unsigned char>, kFields> m_cols;
    View m_view{};
    std::size_t m_slotBytes = 0;
};

template <typename T, typename TDevice = cuda::Device>
class AoSStorage {
    static_assert(std::is_trivially_copyable_v<T>, "graphflow::AoSStorage: payload must be trivially copyable");

public:
    using Payload = T;
    struct View {
        using Payload = T;
        T* data;
        __device__ T load(std::uint64_t slot) const { return data[slot]; }
        __device__ void store(std::uint64_t slot, const T& p) const { data[slot] = p; }
    };

    AoSStorage(const TDevice&, std::uint32_t numChunks, std::uint32_t capacity)
        : m_ledger(numChunks, capacity), m_data(static_cast<std::size_t>(numChunks) * capacity)
    {
    }
    static std::uint64_t slotBytes() { return sizeof(T); }
    View view() const { return View{m_data.data()}; }
    ChunkLedger& ledger() { return m_ledger; }
    const ChunkLedger& ledger() const { return m_ledger; }
    std::uint32_t numChunks() const { return m_ledger.numChunks(); }
    std::uint32_t chunkCapacity() const { return m_ledger.chunkCapacity(); }
    std::uint64_t slotCount() const { return static_cast<std::uint64_t>(numChunks()) * chunkCapacity(); }
    std::uint64_t base(ChunkHandle h) const { return m_ledger.base(h); }

private:
    ChunkLedger m_ledger;
    cuda::Buffer<T> m_data;
};

// flow/PayloadStorage.hpp:946 DefaultStorage: SoA when the payload lists its fields, else AoS.
template <typename T, typename TDevice = cuda::Device>
using DefaultStorage =
    std::conditional_t<requires { SoAFields<T>::count; }, SoAStorage<T, TDevice>, AoSStorage<T, TDevice>>;

} // namespace graphflow
