// C ABI of the hash partition path (16-byte records, SoA or AoS), the device-side plan and the
// record source.
#include <algorithm>
#include <cstdio>

#include "gf_hash.cuh"

bool gf_hash_persistent(); // gf_capi.cu

namespace gf {
namespace {

constexpr int kHashThreads = 256;

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int device_sms()
{
    static int sms = [] {
        int dev = 0, n = 148;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n;
    }();
    return sms;
}

gf_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess)
        return GF_OK;
    std::fprintf(stderr, "graphflow_b200: CUDA error %s\n", cudaGetErrorString(e));
    return GF_ERR_CUDA;
}

template <typename Kernel>
cudaError_t allow_smem(Kernel k, size_t bytes)
{
    if (bytes <= 48u * 1024u)
        return cudaSuccess;
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Grid of a persistent kernel: as many CTAs as fit on the device at once, at most one per tile.
template <typename Kernel>
uint32_t persist_grid(Kernel k, size_t smem, uint32_t n_tiles)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kHashPThreads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const uint64_t g = (uint64_t)per_sm * (uint64_t)device_sms();
    return (uint32_t)std::max<uint64_t>(1u, std::min<uint64_t>(g, n_tiles));
}

template <typename F>
gf_status with_hash_shape(uint32_t tile_size, F&& f)
{
    switch (tile_size) {
    case 1024u:
        return f.template operator()<TileShape<kHashThreads, 4, 2>>();
    case 2048u:
        return f.template operator()<TileShape<kHashThreads, 8, 1>>();
    default:
        return GF_ERR_ARGUMENT;
    }
}

bool cols_ok(const gf_rec16_columns* c, int layout)
{
    if (c == nullptr)
        return false;
    if (layout == GF_LAYOUT_AOS)
        return c->records != nullptr && (reinterpret_cast<uintptr_t>(c->records) & 15u) == 0u;
    if (layout == GF_LAYOUT_SOA)
        return c->key != nullptr && c->weight != nullptr && c->tag != nullptr;
    return false;
}

Rec16SoA soa(const gf_rec16_columns* in, const gf_rec16_columns* out)
{
    Rec16SoA a;
    a.key_in = in ? in->key : nullptr;
    a.w_in = in ? in->weight : nullptr;
    a.tag_in = in ? in->tag : nullptr;
    a.key_out = out ? out->key : nullptr;
    a.w_out = out ? out->weight : nullptr;
    a.tag_out = out ? out->tag : nullptr;
    return a;
}

Rec16AoS aos(const gf_rec16_columns* in, const gf_rec16_columns* out)
{
    Rec16AoS a;
    a.in = in ? static_cast<const Rec16*>(in->records) : nullptr;
    a.out = out ? static_cast<Rec16*>(out->records) : nullptr;
    return a;
}

// Calls f(access) with the access policy of `layout`.
template <typename F>
gf_status with_layout(int layout, const gf_rec16_columns* in, const gf_rec16_columns* out, F&& f)
{
    if (layout == GF_LAYOUT_SOA)
        return f(soa(in, out));
    return f(aos(in, out));
}

} // namespace
} // namespace gf

using namespace gf;

extern "C" {

uint32_t gf_supported_hash_tile_sizes(uint32_t* h_sizes, uint32_t cap)
{
    static const uint32_t sizes[] = {1024u, 2048u};
    for (uint32_t i = 0; i < 2u && i < cap && h_sizes != nullptr; ++i)
        h_sizes[i] = sizes[i];
    return 2u;
}

gf_status gf_classify_hash_r16(void* stream, const gf_rec16_columns* h_cols, int layout, uint32_t capacity,
                               uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size,
                               uint32_t bins, uint64_t salt, uint32_t* d_bin_ids, uint32_t* d_counts,
                               uint32_t* d_status)
{
    if (capacity == 0u || bins == 0u || d_counts == nullptr ||
        (n_tiles != 0u && (d_tiles == nullptr || !cols_ok(h_cols, layout))) ||
        (tile_size != 1024u && tile_size != 2048u))
        return GF_ERR_ARGUMENT;
    if (n_tiles == 0u)
        return GF_OK;
    UnmixClassify cls{salt, bins};
    if (gf_hash_persistent()) {
        return with_layout(layout, h_cols, nullptr, [&](auto acc) -> gf_status {
            using Acc = decltype(acc);
            auto kernel = hash_count_persist_kernel<Acc>;
            const size_t smem = sizeof(uint32_t) * std::min(bins, kHashSmemBins);
            cudaError_t e = allow_smem(kernel, smem);
            if (e != cudaSuccess)
                return cuda_status(e);
            const uint32_t grid = persist_grid(kernel, smem, n_tiles);
            kernel<<<grid, kHashPThreads, smem, as_stream(stream)>>>(acc, cls, capacity, pool_slots, d_tiles, n_tiles,
                                                                    bins, d_bin_ids, d_counts, d_status);
            return cuda_status(cudaGetLastError());
        });
    }
    return with_hash_shape(tile_size, [&]<typename Shape>() -> gf_status {
        return with_layout(layout, h_cols, nullptr, [&](auto acc) -> gf_status {
            using Acc = decltype(acc);
            hash_classify_kernel<Shape, Acc><<<n_tiles, Shape::kThreads, 0, as_stream(stream)>>>(
                acc, cls, capacity, pool_slots, d_tiles, n_tiles, bins, d_bin_ids, d_counts, d_status);
            return cuda_status(cudaGetLastError());
        });
    });
}

gf_status gf_scatter_hash_r16(void* stream, const gf_rec16_columns* h_in, const gf_rec16_columns* h_out, int layout,
                              uint32_t capacity, uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles,
                              uint32_t tile_size, uint32_t bins, uint64_t salt, const uint32_t* d_bin_ids,
                              const uint32_t* d_table, uint32_t* d_next, uint32_t* d_counts, uint32_t* d_status)
{
    if (capacity == 0u || bins == 0u || d_counts == nullptr || d_next == nullptr ||
        (n_tiles != 0u && (d_tiles == nullptr || d_table == nullptr || !cols_ok(h_in, layout) ||
                           !cols_ok(h_out, layout))) ||
        (tile_size != 1024u && tile_size != 2048u))
        return GF_ERR_ARGUMENT;
    if (n_tiles == 0u)
        return GF_OK;
    UnmixClassify cls{salt, bins};
    const FastDiv fdc(capacity);
    if (gf_hash_persistent()) {
        return with_layout(layout, h_in, h_out, [&](auto acc) -> gf_status {
            using Acc = decltype(acc);
            auto kernel = bins > kHashGroupBins     ? hash_scatter_grouped_kernel<Acc, NoUpdate, true, 8u>
                          : bins > kHashGroupBins / 2u ? hash_scatter_grouped_kernel<Acc, NoUpdate, false, 8u>
                                                       : hash_scatter_grouped_kernel<Acc, NoUpdate, false, 4u>;
            const uint32_t unit = tile_size; // 1024 or 2048
            const size_t smem = hash_grouped_smem(bins, unit);
            cudaError_t e = allow_smem(kernel, smem);
            if (e != cudaSuccess)
                return cuda_status(e);
            const uint32_t grid = persist_grid(kernel, smem, n_tiles);
            kernel<<<grid, kHashPThreads, smem, as_stream(stream)>>>(acc, cls, NoUpdate{}, 0u, capacity, fdc,
                                                                    pool_slots, d_tiles, n_tiles, bins, unit, d_bin_ids,
                                                                    d_table, d_next, d_counts, d_status);
            return cuda_status(cudaGetLastError());
        });
    }
    return with_hash_shape(tile_size, [&]<typename Shape>() -> gf_status {
        return with_layout(layout, h_in, h_out, [&](auto acc) -> gf_status {
            using Acc = decltype(acc);
            constexpr int E = 2 * Shape::kTile;
            auto kernel = hash_scatter_kernel<Shape, Acc, NoUpdate>;
            const size_t smem = sizeof(Rec16) * Shape::kTile + sizeof(uint32_t) * Shape::kTile +
                                sizeof(uint32_t) * 4 * E + sizeof(uint32_t) * (Shape::kWarps + 2) + 16;
            cudaError_t e = allow_smem(kernel, smem);
            if (e != cudaSuccess)
                return cuda_status(e);
            kernel<<<n_tiles, Shape::kThreads, smem, as_stream(stream)>>>(acc, cls, NoUpdate{}, 0u, capacity, fdc,
                                                                         pool_slots, d_tiles, n_tiles, bins,
                                                                         d_bin_ids, d_table, d_next, d_counts,
                                                                         d_status);
            return cuda_status(cudaGetLastError());
        });
    });
}

gf_status gf_plan_device(void* stream, const uint32_t* d_counts, uint32_t bins, uint32_t capacity,
                         const uint32_t* d_reserved, uint32_t n_reserved, uint32_t* d_table, gf_out_desc* d_descs,
                         uint32_t desc_cap, uint32_t* d_num_out, uint32_t* d_next, uint32_t* d_status)
{
    if (bins == 0u || capacity == 0u || d_counts == nullptr || d_table == nullptr || d_num_out == nullptr ||
        d_next == nullptr || (n_reserved != 0u && d_reserved == nullptr) || (desc_cap != 0u && d_descs == nullptr))
        return GF_ERR_ARGUMENT;
    const cudaStream_t s = as_stream(stream);
    const FastDiv fdc(capacity);
    const uint32_t n_blocks = (uint32_t)(((uint64_t)bins + kPlanBlock - 1u) / kPlanBlock);
    plan_blocksum_kernel<<<n_blocks, kPlanThreads, 0, s>>>(d_counts, bins, fdc, d_next);
    plan_scan_kernel<1024><<<1, 1024, 0, s>>>(d_counts, bins, n_blocks, n_reserved, desc_cap, d_next, d_num_out,
                                              d_status);
    plan_bins_kernel<<<n_blocks, kPlanThreads, 0, s>>>(d_counts, bins, fdc, n_blocks, d_table, d_next, d_status);
    // one thread per output chunk (at most min(desc_cap, n_reserved) of them), grid-stride
    const uint64_t most = std::max<uint64_t>(std::min<uint64_t>(desc_cap, n_reserved), n_blocks);
    const uint32_t grid = (uint32_t)std::min<uint64_t>((most + kPlanThreads - 1u) / kPlanThreads,
                                                       (uint64_t)device_sms() * 16u);
    plan_chunks_kernel<<<std::max(grid, 1u), kPlanThreads, 0, s>>>(d_counts, bins, capacity, d_reserved, n_blocks,
                                                                   d_table, d_descs, d_num_out, d_next, d_status);
    return cuda_status(cudaGetLastError());
}

gf_status gf_generate_records16(void* stream, uint64_t seed, uint64_t first_id, uint64_t n, const double* d_cdf,
                                uint32_t k, uint64_t salt, const gf_rec16_columns* h_cols, int layout)
{
    if (k == 0u || d_cdf == nullptr || (n != 0u && !cols_ok(h_cols, layout)))
        return GF_ERR_ARGUMENT;
    if (n == 0u)
        return GF_OK;
    const unsigned blocks = (unsigned)((n + 255u) / 256u < 148u * 16u ? (n + 255u) / 256u : 148u * 16u);
    return with_layout(layout, nullptr, h_cols, [&](auto acc) -> gf_status {
        using Acc = decltype(acc);
        generate_records16_kernel<Acc><<<blocks, 256, 0, as_stream(stream)>>>(acc, mix64(seed), first_id, n, d_cdf,
                                                                               k, salt);
        return cuda_status(cudaGetLastError());
    });
}

} // extern "C"
