// Generic C ABI: classify, scatter, transform and the fused partition over the columns of a
// registered record type, with registered classifier, updater and transform functors.
//
// User functors cannot cross a C ABI, so this file is the explicit instantiation table: each
// (record, layout, functor) combination the ids name is a compile-time instantiation of the same
// kernels (gf_partition.cuh, include/graphflow/kernels.cuh) and the same functors
// (examples/particle_feedback.cuh, examples/kernel_axes.cuh) the C++ Flow runs, so a payload
// partitioned through these entry points is partitioned exactly as the Flow partitions it.
// Reference entry points replaced: flow/Execution.hpp:709-776 (TransformKernel), :870-954
// (PartitionClassifyKernel), :985-1189 (PartitionScatterKernel).
#include <string>

#include "../examples/dense_chain.cuh"
#include "../examples/kernel_axes.cuh"
#include "graphflow/kernels.cuh"

void gf_set_last_error(const char* message); // gf_flows.cu

namespace graphflow::generic {

// the one-field records of the registry
struct U32Key {
    std::uint32_t key;
};
struct Rec16 {
    std::uint64_t key;
    float weight;
    std::uint32_t tag;
};

} // namespace graphflow::generic

template <>
struct graphflow::SoAFields<graphflow::generic::U32Key> {
    static constexpr std::size_t count = 1;
    template <typename P, typename F>
    __host__ __device__ static void forEach(P& p, F&& f)
    {
        f(p.key);
    }
};
template <>
struct graphflow::SoAFields<graphflow::generic::Rec16> {
    static constexpr std::size_t count = 3;
    template <typename P, typename F>
    __host__ __device__ static void forEach(P& p, F&& f)
    {
        f(p.key);
        f(p.weight);
        f(p.tag);
    }
};

namespace graphflow::generic {

using particle::Particle;
using dense::KeyRecord;

template <typename T>
constexpr bool kHasKey = requires(const T& p) { p.key; };
template <typename T>
constexpr bool kHasId = requires(const T& p) { p.id; };

// ---- registered classifiers ----
template <typename T>
struct KeyMod { // GF_CLS_KEY_MOD
    std::uint32_t bins;
    __device__ std::uint32_t operator()(const Acc&, const T& p) const
    {
        return static_cast<std::uint32_t>(static_cast<std::uint64_t>(p.key) % bins);
    }
};
template <typename T>
struct IdDistribution { // GF_CLS_ID_* (KernelAxes.hpp:29-42 distributionBin on the id)
    particle::Distribution distribution;
    std::uint32_t bins;
    __device__ std::uint32_t operator()(const Acc&, const T& p) const
    {
        return particle::distributionBin(distribution, static_cast<std::uint64_t>(p.id), bins);
    }
};

// ---- registered transforms ----
struct Identity { // GF_XF_IDENTITY
    template <typename T>
    __device__ void operator()(const Acc&, T&) const
    {
    }
};
struct AddWeight { // GF_XF_ADD_WEIGHT
    std::uint32_t increment;
    __device__ void operator()(const Acc&, Status& st, Particle& p) const
    {
        if (p.weight > 0xFFFFFFFFu - increment) {
            st.set(StatusCode::overflow);
            return;
        }
        p.weight += increment;
        p.visit += 1u;
    }
};

// A pool's view for a record type and layout, built from the caller's columns.
template <typename T, int Layout>
struct ViewOf;
template <typename T>
struct ViewOf<T, GF_LAYOUT_SOA> {
    using View = typename SoAStorage<T>::View;
    static View make(const gf_columns& c)
    {
        View v{};
        for (std::size_t i = 0; i < SoAStorage<T>::kFields; ++i)
            v.cols[i] = static_cast<unsigned char*>(c.column[i]);
        return v;
    }
    static bool complete(const gf_columns& c)
    {
        for (std::size_t i = 0; i < SoAStorage<T>::kFields; ++i)
            if (c.column[i] == nullptr)
                return false;
        return true;
    }
};
template <typename T>
struct ViewOf<T, GF_LAYOUT_AOS> {
    using View = typename AoSStorage<T>::View;
    static View make(const gf_columns& c) { return View{static_cast<T*>(c.column[0])}; }
    static bool complete(const gf_columns& c) { return c.column[0] != nullptr; }
};

// Loads from one view, stores to another (the same columns or another pool of the same record).
template <typename V>
struct InOut {
    using Payload = typename V::Payload;
    V in, out;
    __device__ Payload load(std::uint64_t s) const { return in.load(s); }
    __device__ void store(std::uint64_t s, const Payload& p) const { out.store(s, p); }
};

// Calls f.template operator()<T, Layout>() for the columns' record type and layout.
template <typename F>
gf_status with_record(const gf_columns* c, F&& f)
{
    if (c == nullptr || (c->layout != GF_LAYOUT_SOA && c->layout != GF_LAYOUT_AOS))
        return GF_ERR_ARGUMENT;
    auto go = [&]<typename T>() -> gf_status {
        if (c->layout == GF_LAYOUT_SOA)
            return ViewOf<T, GF_LAYOUT_SOA>::complete(*c) ? f.template operator()<T, GF_LAYOUT_SOA>() : GF_ERR_ARGUMENT;
        return ViewOf<T, GF_LAYOUT_AOS>::complete(*c) ? f.template operator()<T, GF_LAYOUT_AOS>() : GF_ERR_ARGUMENT;
    };
    switch (c->record) {
    case GF_REC_U32:
        return go.template operator()<U32Key>();
    case GF_REC_KEYREC:
        return go.template operator()<KeyRecord>();
    case GF_REC_PARTICLE:
        return go.template operator()<Particle>();
    case GF_REC_R16:
        return go.template operator()<Rec16>();
    default:
        return GF_ERR_ARGUMENT;
    }
}

// Calls f(functor) with the registered classifier `id` for record T (GF_ERR_ARGUMENT if the
// record has no such classifier).
template <typename T, typename F>
gf_status with_classifier(int id, const gf_functor_params& p, std::uint32_t bins, F&& f)
{
    switch (id) {
    case GF_CLS_KEY_MOD:
        if constexpr (kHasKey<T>)
            return f(KeyMod<T>{bins});
        break;
    case GF_CLS_ID_BALANCED:
    case GF_CLS_ID_ONEHOT:
    case GF_CLS_ID_SKEWED:
        if constexpr (kHasId<T>)
            return f(IdDistribution<T>{id == GF_CLS_ID_BALANCED ? particle::Distribution::balanced
                                       : id == GF_CLS_ID_ONEHOT ? particle::Distribution::oneHot
                                                                : particle::Distribution::skewed,
                                       bins});
        break;
    case GF_CLS_FEEDBACK_FILTER:
        if constexpr (std::is_same_v<T, Particle>)
            return f(particle::FilterByProperty{});
        break;
    case GF_CLS_FEEDBACK_SELECT:
        if constexpr (std::is_same_v<T, Particle>)
            return f(particle::SelectOutcome{p.max_visits});
        break;
    default:
        break;
    }
    return GF_ERR_ARGUMENT;
}

// Calls f(updater, bin tag) with the registered updater `id` for record T.
template <typename T, typename F>
gf_status with_updater(int id, const gf_functor_params& p, F&& f)
{
    switch (id) {
    case GF_UPD_NONE:
        return f(NoUpdate{}, std::uint32_t{});
    case GF_UPD_SET_BIN:
        if constexpr (std::is_same_v<T, Particle>)
            return f(particle::KernelBinUpdate{}, std::uint32_t{});
        break;
    case GF_UPD_FEEDBACK:
        if constexpr (std::is_same_v<T, Particle>)
            return f(particle::UpdateWeight{p.increment}, particle::Outcome{});
        break;
    default:
        break;
    }
    return GF_ERR_ARGUMENT;
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

gf_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess)
        return GF_OK;
    gf_set_last_error((std::string("graphflow_b200 generic entry: ") + cudaGetErrorString(e)).c_str());
    return GF_ERR_CUDA;
}

// Shared memory a launch may use on the current device, after opting in.
template <typename K>
gf_status prepare_smem(K kernel, std::size_t bytes)
{
    int dev = 0, limit = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return GF_ERR_CUDA;
    if (bytes > static_cast<std::size_t>(limit)) {
        gf_set_last_error("graphflow_b200 generic entry: the tile of this record and port count needs more "
                          "shared memory per block than the device has");
        return GF_ERR_ARGUMENT;
    }
    if (bytes > 48u * 1024u)
        return cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                static_cast<int>(bytes)));
    return GF_OK;
}

// Calls f.template operator()<Shape>() for the tile size (the dense kernels' 256-thread shapes).
template <typename F>
gf_status with_tile(std::uint32_t tile_size, F&& f)
{
    switch (tile_size) {
    case 1024u:
        return f.template operator()<gf::TileShape<256, 4, 2>>();
    case 2048u:
        return f.template operator()<gf::TileShape<256, 8, 1>>();
    case 4096u:
        return f.template operator()<gf::TileShape<256, 16, 1>>();
    default:
        return GF_ERR_ARGUMENT;
    }
}

template <typename Shape, typename P>
std::size_t scatter_smem(std::uint32_t bins)
{
    return sizeof(P) * Shape::kTile + 4u * Shape::kTile + 4u * Shape::kWarps * bins + 4u * bins * 3u +
           4u * (Shape::kWarps + 2u) + 16u;
}

template <typename Shape, typename P>
std::size_t fused_smem(std::uint32_t bins)
{
    return sizeof(P) * Shape::kTile + 4u * Shape::kTile + 4u * Shape::kWarps * bins + 4u * bins * 6u +
           4u * (2u * Shape::kThreads + Shape::kWarps + 8u);
}

constexpr std::uint32_t kMaxBins = 65535u;

} // namespace graphflow::generic

using namespace graphflow;
using namespace graphflow::generic;

extern "C" gf_status gf_classify_dense(void* stream, const gf_columns* h_cols, uint32_t capacity, uint64_t pool_slots,
                                       const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size, uint32_t bins,
                                       int classifier, const gf_functor_params* h_params, uint32_t* d_bin_ids,
                                       uint32_t* d_counts, uint32_t* d_status)
{
    if (capacity == 0u || bins == 0u || bins > kMaxBins || h_params == nullptr || d_counts == nullptr ||
        (n_tiles != 0u && (d_tiles == nullptr || d_bin_ids == nullptr)))
        return GF_ERR_ARGUMENT;
    return with_record(h_cols, [&]<typename T, int Layout>() -> gf_status {
        using V = typename ViewOf<T, Layout>::View;
        const gf_functor_params prm = *h_params;
        return with_classifier<T>(classifier, prm, bins, [&](auto f) -> gf_status {
            using Cls = ClassifyAdapter<decltype(f), T>;
            const Cls cls{f, gf::mix64(prm.seed), prm.purpose, d_status};
            return with_tile(tile_size, [&]<typename Shape>() -> gf_status {
                if (n_tiles == 0u)
                    return GF_OK;
                auto kernel = gf::classify_kernel<Shape, ViewAccess<V>, Cls>;
                const gf_status rc = prepare_smem(kernel, 4u * bins);
                if (rc != GF_OK)
                    return rc;
                kernel<<<n_tiles, Shape::kThreads, 4u * bins, as_stream(stream)>>>(
                    ViewAccess<V>{ViewOf<T, Layout>::make(*h_cols)}, cls, capacity, pool_slots, d_tiles, n_tiles, bins,
                    d_bin_ids, d_counts, d_status);
                return cuda_status(cudaGetLastError());
            });
        });
    });
}

extern "C" gf_status gf_scatter(void* stream, const gf_columns* h_in, const gf_columns* h_out, uint32_t capacity,
                                uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size,
                                uint32_t bins, const uint32_t* d_bin_ids, const uint32_t* d_table, uint32_t* d_next,
                                uint32_t* d_counts, int mode, int updater, const gf_functor_params* h_params,
                                uint32_t* d_status)
{
    if (capacity == 0u || bins == 0u || bins > kMaxBins || h_params == nullptr || h_in == nullptr ||
        h_out == nullptr || h_in->record != h_out->record || h_in->layout != h_out->layout || d_counts == nullptr ||
        d_next == nullptr || (mode != GF_SCATTER_SHARED && mode != GF_SCATTER_DIRECT) ||
        (n_tiles != 0u && (d_tiles == nullptr || d_bin_ids == nullptr || d_table == nullptr)))
        return GF_ERR_ARGUMENT;
    return with_record(h_in, [&]<typename T, int Layout>() -> gf_status {
        using V = typename ViewOf<T, Layout>::View;
        if (!ViewOf<T, Layout>::complete(*h_out))
            return GF_ERR_ARGUMENT;
        const gf_functor_params prm = *h_params;
        const InOut<V> acc{ViewOf<T, Layout>::make(*h_in), ViewOf<T, Layout>::make(*h_out)};
        return with_updater<T>(updater, prm, [&](auto u, auto bin_tag) -> gf_status {
            using Upd = UpdateAdapter<decltype(u), decltype(bin_tag), T>;
            const Upd upd{u, prm.purpose + 1u, d_status};
            const std::uint64_t seed_mixed = gf::mix64(prm.seed);
            return with_tile(tile_size, [&]<typename Shape>() -> gf_status {
                if (n_tiles == 0u)
                    return GF_OK;
                const gf::FastDiv fdc(capacity);
                if (mode == GF_SCATTER_DIRECT) {
                    auto kernel = gf::scatter_direct_kernel<Shape, InOut<V>, Upd>;
                    kernel<<<n_tiles, Shape::kThreads, 0, as_stream(stream)>>>(
                        acc, upd, seed_mixed, capacity, fdc, pool_slots, d_tiles, n_tiles, bins, d_bin_ids, d_table,
                        d_next, d_counts, d_status);
                    return cuda_status(cudaGetLastError());
                }
                auto kernel = gf::scatter_kernel<Shape, InOut<V>, Upd>;
                const std::size_t smem = scatter_smem<Shape, T>(bins);
                const gf_status rc = prepare_smem(kernel, smem);
                if (rc != GF_OK)
                    return rc;
                kernel<<<n_tiles, Shape::kThreads, smem, as_stream(stream)>>>(acc, upd, seed_mixed, capacity, fdc,
                                                                             pool_slots, d_tiles, n_tiles, bins,
                                                                             d_bin_ids, d_table, d_next, d_counts,
                                                                             d_status);
                return cuda_status(cudaGetLastError());
            });
        });
    });
}

extern "C" gf_status gf_transform(void* stream, const gf_columns* h_in, const gf_columns* h_out, uint32_t capacity,
                                  uint64_t pool_slots, const gf_move_tile* d_tiles, uint32_t n_tiles,
                                  const uint32_t* d_out_chunks, uint32_t n_out, int transform,
                                  const gf_functor_params* h_params, uint32_t* d_status)
{
    static_assert(sizeof(gf_move_tile) == sizeof(MoveTile), "gf_move_tile is MoveTile");
    if (capacity == 0u || h_params == nullptr || h_in == nullptr || h_out == nullptr ||
        h_in->record != h_out->record || h_in->layout != h_out->layout ||
        (n_tiles != 0u && (d_tiles == nullptr || d_out_chunks == nullptr)))
        return GF_ERR_ARGUMENT;
    return with_record(h_in, [&]<typename T, int Layout>() -> gf_status {
        using V = typename ViewOf<T, Layout>::View;
        if (!ViewOf<T, Layout>::complete(*h_out))
            return GF_ERR_ARGUMENT;
        const gf_functor_params prm = *h_params;
        const InOut<V> view{ViewOf<T, Layout>::make(*h_in), ViewOf<T, Layout>::make(*h_out)};
        auto launch = [&](auto f) -> gf_status {
            if (n_tiles == 0u)
                return GF_OK;
            const unsigned grid = n_tiles < 65535u ? n_tiles : 65535u;
            transform_kernel<<<grid, 256, 0, as_stream(stream)>>>(
                f, view, gf::mix64(prm.seed), prm.purpose, reinterpret_cast<const MoveTile*>(d_tiles), n_tiles,
                d_out_chunks, n_out, capacity, gf::FastDiv(capacity), pool_slots, d_status);
            return cuda_status(cudaGetLastError());
        };
        if (transform == GF_XF_IDENTITY)
            return launch(Identity{});
        if constexpr (std::is_same_v<T, Particle>)
            if (transform == GF_XF_ADD_WEIGHT)
                return launch(AddWeight{prm.increment});
        return GF_ERR_ARGUMENT;
    });
}

extern "C" gf_status gf_partition_fused(void* stream, const gf_columns* h_cols, uint32_t capacity,
                                        uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t bins,
                                        int classifier, int updater, const gf_functor_params* h_params,
                                        const uint32_t* d_reserved, uint32_t n_reserved, uint32_t* d_totals,
                                        unsigned long long* d_port_chunks, uint32_t max_chunks_per_port,
                                        void* d_scratch, uint64_t scratch_bytes, uint32_t* d_table,
                                        gf_out_desc* d_descs, uint32_t desc_cap, uint32_t* d_num_out,
                                        uint32_t* d_status)
{
    using Shape = gf::TileShape<256, 4, 2>; // tiles of 1024, as the Flow's partition stage
    uint64_t need = 0;
    if (capacity == 0u || bins == 0u || bins > kMaxBins || h_params == nullptr || d_totals == nullptr ||
        d_status == nullptr || d_table == nullptr || d_num_out == nullptr || (desc_cap != 0u && d_descs == nullptr) ||
        gf_fused_scratch_bytes(n_tiles, bins, &need) != GF_OK || scratch_bytes < need || d_scratch == nullptr ||
        (reinterpret_cast<uintptr_t>(d_scratch) & 15u) != 0u ||
        (n_tiles != 0u && (d_tiles == nullptr || d_port_chunks == nullptr || max_chunks_per_port == 0u)))
        return GF_ERR_ARGUMENT;
    return with_record(h_cols, [&]<typename T, int Layout>() -> gf_status {
        using V = typename ViewOf<T, Layout>::View;
        const gf_functor_params prm = *h_params;
        return with_classifier<T>(classifier, prm, bins, [&](auto f) -> gf_status {
            using Cls = ClassifyAdapter<decltype(f), T>;
            const Cls cls{f, gf::mix64(prm.seed), prm.purpose, d_status};
            return with_updater<T>(updater, prm, [&](auto u, auto bin_tag) -> gf_status {
                using Upd = UpdateAdapter<decltype(u), decltype(bin_tag), T>;
                const Upd upd{u, prm.purpose + 1u, d_status};
                auto* ctl = static_cast<gf::FusedCtl*>(d_scratch);
                if (n_tiles == 0u) {
                    cudaError_t e = cudaMemsetAsync(d_totals, 0, sizeof(uint32_t) * bins, as_stream(stream));
                    if (e != cudaSuccess)
                        return cuda_status(e);
                    return gf_fused_finish(stream, d_totals, d_port_chunks, bins, capacity, max_chunks_per_port,
                                           d_scratch, d_table, d_descs, desc_cap, d_num_out, d_status);
                }
                auto kernel = gf::fused_partition_kernel<Shape, ViewAccess<V>, Cls, Upd>;
                const std::size_t smem = fused_smem<Shape, T>(bins);
                gf_status rc = prepare_smem(kernel, smem);
                if (rc != GF_OK)
                    return rc;
                cudaError_t e = cudaMemsetAsync(ctl, 0, gf::kFusedCtlResetBytes, as_stream(stream));
                if (e != cudaSuccess)
                    return cuda_status(e);
                kernel<<<n_tiles, Shape::kThreads, smem, as_stream(stream)>>>(
                    ViewAccess<V>{ViewOf<T, Layout>::make(*h_cols)}, cls, upd, gf::mix64(prm.seed), capacity,
                    gf::FastDiv(capacity), pool_slots, d_tiles, n_tiles, bins, d_reserved, n_reserved, d_totals,
                    d_port_chunks, max_chunks_per_port, ctl, reinterpret_cast<unsigned long long*>(ctl + 1), d_status,
                    gf::InlineFinish{d_table, d_descs, desc_cap, d_num_out}, gf::NoPost{});
                return cuda_status(cudaGetLastError());
            });
        });
    });
}
