// C ABI of the dense partition kernels and the synthetic key source: argument validation on the
// host, then dispatch to the tile-size instantiations of gf_partition.cuh.
#include <cstdio>
#include <algorithm>
#include <mutex>
#include <string>

#include "gf_fused_bulk.cuh"
#include "gf_fused_coop.cuh"

namespace gf {
namespace {

// Tuning knob: 1 = gf_partition_fused_u32 uses the cooperative count/plan/scatter kernel where it
// applies (default); 0 = always the per-tile look-back kernel.
int g_fused_coop = 1;
// Tuning knob: 1 = for up to 16 ports the cooperative kernel writes tiles out with bulk copies
// (fused_partition_coop_bulk_kernel) when the scratch holds its tile histograms (default); 0 = the
// warp-store write-out of fused_partition_coop_kernel for every port count.
int g_fused_coop_bulk = 1;
// Tuning knob: 1 = the flow entry points run the B200 runner options (sinks take up to Q chunks,
// every idle node is dispatched per loop iteration); 0 = the reference's one-chunk sinks and one
// dispatch per iteration.
int g_runner_batched = 1;
// Tuning knob: 1 = the hash classify/scatter entry points use the persistent kernels (one shared
// counter per port and CTA); 0 = the per-tile open-addressing kernels.
int g_hash_persistent = 1;
int g_sink_batch = 256;
// Tuning knob: 1 = with the B200 runner options, the fused partition nodes of one type run as one
// partition group (one multi-batch launch drains every member's ready batches); 0 = one runner node
// per partition node.
int g_group_partitions = 1;
// Tuning knob: 1 = the flow entry points run their Flow device-resident (Tuning::deviceResident:
// waves of whole-list batches on one stream with a device chunk pool); 0 = the host runner (default).
int g_device_resident = 0;
// Tuning knob: 1 = device-resident partition batches of at least 64 tiles and up to 64 ports run the
// cooperative kernel of gf_fused_any.cuh (default); 0 = always the per-tile look-back kernel.
int g_device_coop = 1;

constexpr int kThreads = 256;
constexpr uint32_t kMaxDenseBins = 65535u;

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

gf_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess)
        return GF_OK;
    std::fprintf(stderr, "graphflow_b200: CUDA error %s\n", cudaGetErrorString(e));
    return GF_ERR_CUDA;
}

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

template <typename Kernel>
cudaError_t allow_smem(Kernel k, size_t bytes)
{
    if (bytes <= 48u * 1024u)
        return cudaSuccess;
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename Shape, typename P>
size_t staged_smem(uint32_t B, uint32_t extra_bin_arrays)
{
    return sizeof(P) * Shape::kTile + sizeof(uint32_t) * Shape::kTile + sizeof(uint32_t) * Shape::kWarps * B +
           sizeof(uint32_t) * B * extra_bin_arrays + sizeof(uint32_t) * (Shape::kWarps + 2) + 16;
}

bool valid_tile_size(uint32_t t) { return t == 1024u || t == 2048u || t == 4096u || t == 8192u; }

// Calls f.template operator()<Shape>() for the instantiation of `tile_size`.
template <typename F>
gf_status with_shape(uint32_t tile_size, F&& f)
{
    switch (tile_size) {
    case 1024u:
        return f.template operator()<TileShape<kThreads, 4, 4>>();
    case 2048u:
        return f.template operator()<TileShape<kThreads, 8, 3>>();
    case 4096u:
        return f.template operator()<TileShape<kThreads, 16, 3>>();
    case 8192u:
        return f.template operator()<TileShape<kThreads, 32, 1>>();
    default:
        return GF_ERR_ARGUMENT;
    }
}

KeyClassifier key_classifier(int cls, uint32_t bins)
{
    KeyClassifier k;
    k.kind = cls;
    k.bins = bins;
    k.fd = FastDiv(bins);
    k.salt = 0u;
    return k;
}

bool valid_classifier(int cls)
{
    return cls == GF_CLS_KEY_MOD || cls == GF_CLS_ID_BALANCED || cls == GF_CLS_ID_ONEHOT || cls == GF_CLS_ID_SKEWED;
}

} // namespace
} // namespace gf

using namespace gf;

extern "C" {

gf_status gf_set_tuning(const char* name, int value)
{
    if (name == nullptr)
        return GF_ERR_ARGUMENT;
    if (std::string(name) == "fused_coop") {
        g_fused_coop = value != 0;
        return GF_OK;
    }
    if (std::string(name) == "fused_coop_bulk") {
        g_fused_coop_bulk = value != 0;
        return GF_OK;
    }
    if (std::string(name) == "runner_batched") {
        g_runner_batched = value != 0;
        return GF_OK;
    }
    if (std::string(name) == "group_partitions") {
        g_group_partitions = value != 0;
        return GF_OK;
    }
    if (std::string(name) == "device_resident") {
        g_device_resident = value != 0;
        return GF_OK;
    }
    if (std::string(name) == "device_coop") {
        g_device_coop = value != 0;
        return GF_OK;
    }
    if (std::string(name) == "hash_persistent") {
        g_hash_persistent = value != 0;
        return GF_OK;
    }
    if (std::string(name) == "spin_limit") {
        // polls a wait between CTAs of the dense fused partition entry points makes before it gives
        // up with GF_ERR_TIMEOUT; <= 0 restores the default (a synchronous 4-byte copy to the device)
        const uint32_t v = value <= 0 ? kSpinLimit : (uint32_t)value;
        return cuda_status(cudaMemcpyToSymbol(g_spin_limit, &v, sizeof(v)));
    }
    if (std::string(name) == "sink_batch_chunks") {
        if (value < 1 || value > 256)
            return GF_ERR_ARGUMENT;
        g_sink_batch = value;
        return GF_OK;
    }
    return GF_ERR_ARGUMENT;
}

uint32_t gf_supported_tile_sizes(uint32_t* h_sizes, uint32_t cap)
{
    static const uint32_t sizes[] = {1024u, 2048u, 4096u, 8192u};
    for (uint32_t i = 0; i < 4u && i < cap && h_sizes != nullptr; ++i)
        h_sizes[i] = sizes[i];
    return 4u;
}

gf_status gf_classify_dense_u32(void* stream, const uint32_t* d_keys, uint32_t capacity, uint64_t pool_slots,
                                const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size, uint32_t bins,
                                int classifier, uint32_t* d_bin_ids, uint32_t* d_counts, uint32_t* d_status)
{
    if (capacity == 0u || bins == 0u || bins > kMaxDenseBins || !valid_tile_size(tile_size) ||
        !valid_classifier(classifier) || d_counts == nullptr || (n_tiles != 0u && (d_keys == nullptr ||
                                                                                    d_tiles == nullptr ||
                                                                                    d_bin_ids == nullptr)))
        return GF_ERR_ARGUMENT;
    if (n_tiles == 0u)
        return GF_OK;
    return with_shape(tile_size, [&]<typename Shape>() -> gf_status {
        using Acc = U32Column;
        auto kernel = classify_kernel<Shape, Acc, KeyClassify<Acc>>;
        const size_t smem = sizeof(uint32_t) * bins;
        cudaError_t e = allow_smem(kernel, smem);
        if (e != cudaSuccess)
            return cuda_status(e);
        Acc acc{d_keys, nullptr};
        KeyClassify<Acc> cls{key_classifier(classifier, bins)};
        kernel<<<n_tiles, Shape::kThreads, smem, as_stream(stream)>>>(
            acc, cls, capacity, pool_slots, d_tiles, n_tiles, bins, d_bin_ids, d_counts, d_status);
        return cuda_status(cudaGetLastError());
    });
}

gf_status gf_scatter_dense_u32(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out, uint32_t capacity,
                               uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size,
                               uint32_t bins, const uint32_t* d_bin_ids, const uint32_t* d_table, uint32_t* d_next,
                               uint32_t* d_counts, int mode, uint32_t* d_status)
{
    if (capacity == 0u || bins == 0u || bins > kMaxDenseBins || !valid_tile_size(tile_size) ||
        (mode != GF_SCATTER_SHARED && mode != GF_SCATTER_DIRECT) || d_counts == nullptr || d_next == nullptr ||
        (n_tiles != 0u && (d_keys_in == nullptr || d_keys_out == nullptr || d_tiles == nullptr ||
                           d_bin_ids == nullptr || d_table == nullptr)))
        return GF_ERR_ARGUMENT;
    if (n_tiles == 0u)
        return GF_OK;
    return with_shape(tile_size, [&]<typename Shape>() -> gf_status {
        using Acc = U32Column;
        Acc acc{d_keys_in, d_keys_out};
        const FastDiv fdc(capacity);
        if (mode == GF_SCATTER_DIRECT) {
            auto kernel = scatter_direct_kernel<Shape, Acc, NoUpdate>;
            kernel<<<n_tiles, Shape::kThreads, 0, as_stream(stream)>>>(acc, NoUpdate{}, 0u, capacity, fdc,
                                                                        pool_slots, d_tiles, n_tiles, bins,
                                                                        d_bin_ids, d_table, d_next, d_counts,
                                                                        d_status);
            return cuda_status(cudaGetLastError());
        }
        auto kernel = scatter_kernel<Shape, Acc, NoUpdate>;
        const size_t smem = staged_smem<Shape, uint32_t>(bins, 3u);
        cudaError_t e = allow_smem(kernel, smem);
        if (e != cudaSuccess)
            return cuda_status(e);
        kernel<<<n_tiles, Shape::kThreads, smem, as_stream(stream)>>>(
            acc, NoUpdate{}, 0u, capacity, fdc, pool_slots, d_tiles, n_tiles, bins, d_bin_ids, d_table, d_next,
            d_counts, d_status);
        return cuda_status(cudaGetLastError());
    });
}

gf_status gf_fused_scratch_bytes(uint32_t n_tiles, uint32_t bins, uint64_t* h_bytes)
{
    if (h_bytes == nullptr || bins == 0u)
        return GF_ERR_ARGUMENT;
    // at least four ports' worth per tile: room for the cooperative kernels' tile histograms
    *h_bytes = sizeof(FusedCtl) + (uint64_t)n_tiles * std::max(bins, 4u) * sizeof(unsigned long long);
    return GF_OK;
}

} // extern "C"

namespace {
// The fused partition; with `fin` set, the same launch also writes gf_fused_finish's outputs (the
// cooperative kernel during its plan, the per-tile kernel in its last CTA). `finished` reports
// whether it did (false only for an empty batch).
gf_status fused_u32(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out, uint32_t capacity,
                    uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size, uint32_t bins,
                    int classifier, const uint32_t* d_reserved, uint32_t n_reserved, uint32_t* d_totals,
                    unsigned long long* d_port_chunks, uint32_t max_chunks_per_port, void* d_scratch,
                    uint64_t scratch_bytes, uint32_t* d_status, InlineFinish fin, bool* finished)
{
    *finished = false;
    uint64_t need = 0;
    if (gf_fused_scratch_bytes(n_tiles, bins, &need) != GF_OK || scratch_bytes < need || d_scratch == nullptr ||
        (reinterpret_cast<uintptr_t>(d_scratch) & 15u) != 0u)
        return GF_ERR_ARGUMENT;
    if (capacity == 0u || bins > kMaxDenseBins || !valid_tile_size(tile_size) || !valid_classifier(classifier) ||
        d_totals == nullptr || d_status == nullptr ||
        (n_tiles != 0u && (d_keys_in == nullptr || d_keys_out == nullptr || d_tiles == nullptr ||
                           d_port_chunks == nullptr || max_chunks_per_port == 0u)))
        return GF_ERR_ARGUMENT;
    if (n_tiles == 0u)
        return cuda_status(cudaMemsetAsync(d_totals, 0, sizeof(uint32_t) * bins, as_stream(stream)));
    *finished = fin.table != nullptr;
    FusedCtl* ctl = static_cast<FusedCtl*>(d_scratch);
    unsigned long long* desc = reinterpret_cast<unsigned long long*>(ctl + 1);
    const bool coop = g_fused_coop != 0 && bins <= 64u && (capacity & 3u) == 0u && capacity >= 4096u &&
                      tile_size <= 4096u && pool_slots < 0xFFFFFFFFull && (reinterpret_cast<uintptr_t>(d_keys_in) & 15u) == 0u &&
                      (reinterpret_cast<uintptr_t>(d_keys_out) & 15u) == 0u &&
                      scratch_bytes >= sizeof(FusedCtl) + sizeof(CoopHdr) + 256u;
    if (coop) {
        // the cooperative control block and the per-CTA port totals live in the descriptor area of
        // the scratch; the launcher zeroes the control block's reset words
        auto launch = [&]<typename S, typename Cls>(Cls cls) -> gf_status {
            if constexpr (requires { S::kHistWords; })
                return cuda_status(launch_fused_coop_bulk<S>(
                    as_stream(stream), cls, d_keys_in, d_keys_out, capacity, pool_slots, d_tiles, n_tiles, bins,
                    d_reserved, n_reserved, d_totals, d_port_chunks, max_chunks_per_port, ctl, scratch_bytes,
                    d_status, device_sms(), fin));
            else
                return cuda_status(launch_fused_coop<S>(as_stream(stream), cls, d_keys_in, d_keys_out, capacity,
                                                        pool_slots, d_tiles, n_tiles, bins, d_reserved, n_reserved,
                                                        d_totals, d_port_chunks, max_chunks_per_port, ctl,
                                                        scratch_bytes, d_status, device_sms(), fin));
        };
        auto with_cls = [&]<typename S>() -> gf_status {
            if (classifier == GF_CLS_KEY_MOD || classifier == GF_CLS_ID_BALANCED) {
                if ((bins & (bins - 1u)) == 0u)
                    return launch.template operator()<S>(MaskClassify{bins - 1u});
                return launch.template operator()<S>(ModClassify{FastDiv(bins)});
            }
            return launch.template operator()<S>(AnyKeyClassify{key_classifier(classifier, bins)});
        };
        const int sms = device_sms();
        if (bins <= 4u && g_fused_coop_bulk != 0 && coop_bulk_fits<CoopBulkShape<2>>(n_tiles, scratch_bytes, sms))
            return with_cls.template operator()<CoopBulkShape<2>>();
        if (bins <= 4u)
            return with_cls.template operator()<CoopShape<2>>();
        if (bins <= 16u && g_fused_coop_bulk != 0 && coop_bulk_fits<CoopBulkShape<8>>(n_tiles, scratch_bytes, sms))
            return with_cls.template operator()<CoopBulkShape<8>>();
        if (bins <= 16u)
            return with_cls.template operator()<CoopShape<8>>();
        return with_cls.template operator()<CoopShape<32>>();
    }
    cudaError_t e = cudaMemsetAsync(ctl, 0, kFusedCtlResetBytes, as_stream(stream));
    if (e != cudaSuccess)
        return cuda_status(e);
    return with_shape(tile_size, [&]<typename Shape>() -> gf_status {
        using Acc = U32Column;
        auto kernel = fused_partition_kernel<Shape, Acc, KeyClassify<Acc>, NoUpdate>;
        const size_t smem = staged_smem<Shape, uint32_t>(bins, 6u) + sizeof(uint32_t) * (4 + 2 * Shape::kThreads);
        cudaError_t err = allow_smem(kernel, smem);
        if (err != cudaSuccess)
            return cuda_status(err);
        Acc acc{d_keys_in, d_keys_out};
        KeyClassify<Acc> cls{key_classifier(classifier, bins)};
        kernel<<<n_tiles, Shape::kThreads, smem, as_stream(stream)>>>(
            acc, cls, NoUpdate{}, 0u, capacity, FastDiv(capacity), pool_slots, d_tiles, n_tiles, bins, d_reserved,
            n_reserved, d_totals, d_port_chunks, max_chunks_per_port, ctl, desc, d_status, fin, NoPost{});
        return cuda_status(cudaGetLastError());
    });
}
} // namespace

extern "C" {

gf_status gf_partition_fused_u32(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out, uint32_t capacity,
                                 uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size,
                                 uint32_t bins, int classifier, const uint32_t* d_reserved, uint32_t n_reserved,
                                 uint32_t* d_totals, unsigned long long* d_port_chunks, uint32_t max_chunks_per_port,
                                 void* d_scratch, uint64_t scratch_bytes, uint32_t* d_status)
{
    bool finished = false;
    return fused_u32(stream, d_keys_in, d_keys_out, capacity, pool_slots, d_tiles, n_tiles, tile_size, bins,
                     classifier, d_reserved, n_reserved, d_totals, d_port_chunks, max_chunks_per_port, d_scratch,
                     scratch_bytes, d_status, InlineFinish{}, &finished);
}

gf_status gf_partition_fused_full_u32(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out,
                                      uint32_t capacity, uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles,
                                      uint32_t tile_size, uint32_t bins, int classifier, const uint32_t* d_reserved,
                                      uint32_t n_reserved, uint32_t* d_totals, unsigned long long* d_port_chunks,
                                      uint32_t max_chunks_per_port, void* d_scratch, uint64_t scratch_bytes,
                                      uint32_t* d_table, gf_out_desc* d_descs, uint32_t desc_cap,
                                      uint32_t* d_num_out, uint32_t* d_status)
{
    if (d_table == nullptr || d_num_out == nullptr || (desc_cap != 0u && d_descs == nullptr))
        return GF_ERR_ARGUMENT;
    bool finished = false;
    const gf_status rc = fused_u32(stream, d_keys_in, d_keys_out, capacity, pool_slots, d_tiles, n_tiles, tile_size,
                                   bins, classifier, d_reserved, n_reserved, d_totals, d_port_chunks,
                                   max_chunks_per_port, d_scratch, scratch_bytes, d_status,
                                   InlineFinish{d_table, d_descs, desc_cap, d_num_out}, &finished);
    if (rc != GF_OK || finished)
        return rc;
    return gf_fused_finish(stream, d_totals, d_port_chunks, bins, capacity, max_chunks_per_port, d_scratch, d_table,
                           d_descs, desc_cap, d_num_out, d_status);
}

gf_status gf_fused_finish(void* stream, const uint32_t* d_totals, const unsigned long long* d_port_chunks,
                          uint32_t bins, uint32_t capacity, uint32_t max_chunks_per_port, const void* d_scratch,
                          uint32_t* d_table, gf_out_desc* d_descs, uint32_t desc_cap, uint32_t* d_num_out,
                          uint32_t* d_status)
{
    if (bins == 0u || capacity == 0u || d_totals == nullptr || d_table == nullptr || d_num_out == nullptr ||
        d_scratch == nullptr ||
        (desc_cap != 0u && (d_descs == nullptr || d_port_chunks == nullptr)))
        return GF_ERR_ARGUMENT;
    constexpr int T = 1024;
    const size_t smem = sizeof(uint32_t) * (4096u * 2u + T / 32 + 1);
    cudaError_t e = allow_smem(fused_finish_kernel<T>, smem);
    if (e != cudaSuccess)
        return cuda_status(e);
    fused_finish_kernel<T><<<1, T, smem, as_stream(stream)>>>(d_totals, d_port_chunks, bins, capacity,
                                                              FastDiv(capacity), max_chunks_per_port,
                                                              static_cast<const FusedCtl*>(d_scratch), d_table,
                                                              d_descs, desc_cap, d_num_out, d_status);
    return cuda_status(cudaGetLastError());
}

gf_status gf_generate_keys_u32(void* stream, int dist, uint64_t seed, uint64_t first_id, uint64_t n, uint32_t bins,
                               const double* d_cdf, uint32_t* d_keys)
{
    if (dist < GF_DIST_UNIFORM || dist > GF_DIST_ROUND_ROBIN || (dist == GF_DIST_ZIPF && (d_cdf == nullptr ||
                                                                                       bins == 0u)) ||
        (n != 0u && d_keys == nullptr))
        return GF_ERR_ARGUMENT;
    if (n == 0u)
        return GF_OK;
    const uint64_t blocks64 = (n + 255u) / 256u;
    const unsigned blocks = (unsigned)(blocks64 < (uint64_t)device_sms() * 16u ? blocks64 : (uint64_t)device_sms() * 16u);
    generate_keys_kernel<<<blocks, 256, 0, as_stream(stream)>>>(dist, mix64(seed), first_id, n, bins, d_cdf, d_keys);
    return cuda_status(cudaGetLastError());
}

} // extern "C"

// ---------------------------------------------------------------------------------------------
// Fused partition without device allocation.
//
// For callers that cannot allocate device memory when they partition: a host runtime that hands
// all device memory to its own pool at start-up and forbids cudaMalloc afterwards, or a
// latency-critical path where cudaMalloc/cudaFree (which can synchronise the device) are not
// acceptable. Their scratch (control block + per-(tile, port) look-back descriptors) lives in the
// file-scope array below, sized kNoAllocScratchBytes, which every GPU that loads this library
// holds until the process exits.
// ---------------------------------------------------------------------------------------------
void gf_set_last_error(const char* message); // gf_flows.cu

namespace {

constexpr uint64_t kNoAllocScratchBytes = 8ull << 20; // 8 MiB
constexpr int kNoAllocMaxDevices = 64;

// Host code must never pass this name to a kernel: on the host it is only a stand-in for the
// device array. Its device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::once_flag g_noalloc_once[kNoAllocMaxDevices];
void* g_noalloc_ptr[kNoAllocMaxDevices];
cudaError_t g_noalloc_err[kNoAllocMaxDevices];

// Set-up of the current device, done by its first call: take the array's device address and
// zero the control block (a 64-byte synchronous cudaMemset; it allocates nothing). The address is
// kept for the life of the process's primary context on that device.
void* noalloc_scratch(gf_status* rc)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *rc = cuda_status(e);
        return nullptr;
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        gf_set_last_error(("gf_partition_fused_u32_noalloc: device " + std::to_string(dev) +
                           " is beyond the " + std::to_string(kNoAllocMaxDevices) + " devices it serves")
                              .c_str());
        *rc = GF_ERR_RANGE;
        return nullptr;
    }
    std::call_once(g_noalloc_once[dev], [dev] {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err == cudaSuccess)
            err = cudaMemset(p, 0, sizeof(FusedCtl));
        g_noalloc_ptr[dev] = err == cudaSuccess ? p : nullptr;
        g_noalloc_err[dev] = err;
    });
    if (g_noalloc_err[dev] != cudaSuccess) {
        *rc = cuda_status(g_noalloc_err[dev]);
        return nullptr;
    }
    *rc = GF_OK;
    return g_noalloc_ptr[dev];
}

} // namespace

extern "C" gf_status gf_partition_fused_u32_noalloc(
    void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out, uint32_t capacity, uint64_t pool_slots,
    const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size, uint32_t bins, int classifier,
    const uint32_t* d_reserved, uint32_t n_reserved, uint32_t* d_totals, unsigned long long* d_port_chunks,
    uint32_t max_chunks_per_port, uint32_t* d_table, gf_out_desc* d_descs, uint32_t desc_cap, uint32_t* d_num_out,
    uint32_t* d_status)
{
    uint64_t need = 0;
    if (gf_fused_scratch_bytes(n_tiles, bins, &need) != GF_OK)
        return GF_ERR_ARGUMENT;
    if (need > kNoAllocScratchBytes) {
        gf_set_last_error(("gf_partition_fused_u32_noalloc: the batch needs " + std::to_string(need) +
                           " scratch bytes (64 + 8 x tiles x max(ports, 4)) but the static scratch holds " +
                           std::to_string(kNoAllocScratchBytes) + "; use gf_partition_fused_u32 with caller scratch")
                              .c_str());
        return GF_ERR_RANGE;
    }
    // the finish outputs are checked before anything runs, so a bad argument changes no output
    if (d_table == nullptr || d_num_out == nullptr || (desc_cap != 0u && d_descs == nullptr))
        return GF_ERR_ARGUMENT;
    gf_status rc = GF_OK;
    void* scratch = noalloc_scratch(&rc);
    if (scratch == nullptr)
        return rc;
    // partition and finish in one launch where the kernel allows it (same results as the two calls)
    return gf_partition_fused_full_u32(stream, d_keys_in, d_keys_out, capacity, pool_slots, d_tiles, n_tiles,
                                       tile_size, bins, classifier, d_reserved, n_reserved, d_totals, d_port_chunks,
                                       max_chunks_per_port, scratch, kNoAllocScratchBytes, d_table, d_descs, desc_cap,
                                       d_num_out, d_status);
}

// Read by the flow entry points (gf_flows.cu, gf_dense_flow.cu, gf_photon.cu).
bool gf_runner_batched() { return gf::g_runner_batched != 0; }
// Chunks a sink takes per launch in the batched runner (gf_flows.cu, gf_dense_flow.cu, gf_photon.cu).
uint32_t gf_runner_sink_batch() { return (uint32_t)gf::g_sink_batch; }
// Read by the flow entry points (gf_dense_flow.cu, gf_flows.cu).
bool gf_group_partitions() { return gf::g_group_partitions != 0; }
bool gf_device_resident() { return gf::g_device_resident != 0; }
bool gf_device_coop() { return gf::g_device_coop != 0; }
// Read by the hash entry points (gf_capi_hash.cu).
bool gf_hash_persistent() { return gf::g_hash_persistent != 0; }
