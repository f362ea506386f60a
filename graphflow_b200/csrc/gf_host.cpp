// Host-side planning entry points of the C ABI: reservation bound, dense plan, dense table,
// tile flattening and the Zipf table of the synthetic sources. Plain C++ (no device work).
#include <cmath>
#include <cstdint>
#include <limits>

#include "graphflow_b200.h"

namespace {

bool ceil_div(uint64_t num, uint64_t den, uint64_t& out)
{
    if (den == 0u)
        return false;
    out = num / den + (num % den != 0u ? 1u : 0u);
    return true;
}

} // namespace

extern "C" {

// core/Reservation.hpp:35-50
gf_status gf_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint64_t* h_out)
{
    if (h_out == nullptr)
        return GF_ERR_ARGUMENT;
    if (n == 0u) {
        *h_out = 0u;
        return GF_OK;
    }
    if (capacity == 0u || max_bins == 0u)
        return GF_ERR_ARGUMENT;
    uint64_t per_chunk = 0;
    ceil_div(n, capacity, per_chunk);
    const uint64_t bins = max_bins < n ? max_bins : n;
    if (per_chunk > std::numeric_limits<uint64_t>::max() - bins + 1u)
        return GF_ERR_RANGE;
    const uint64_t bound = per_chunk + bins - 1u;
    *h_out = bound < n ? bound : n;
    return GF_OK;
}

// core/Reservation.hpp:61-71
gf_status gf_checked_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint32_t* h_out)
{
    if (h_out == nullptr)
        return GF_ERR_ARGUMENT;
    uint64_t b = 0;
    const gf_status rc = gf_output_chunk_bound(n, capacity, max_bins, &b);
    if (rc != GF_OK)
        return rc;
    if (b > std::numeric_limits<uint32_t>::max())
        return GF_ERR_RANGE;
    *h_out = static_cast<uint32_t>(b);
    return GF_OK;
}

// graph/DenseBinTable.hpp:39-77
gf_status gf_plan_dense(const uint32_t* h_totals, uint32_t bins, uint32_t capacity, uint32_t* h_bin_base,
                        uint32_t* h_fills, uint32_t fills_cap, uint32_t* h_num_out)
{
    if (bins == 0u || capacity == 0u || h_totals == nullptr || h_bin_base == nullptr || h_num_out == nullptr)
        return GF_ERR_ARGUMENT;
    uint64_t exact = 0u, particles = 0u;
    for (uint32_t b = 0; b < bins; ++b) {
        h_bin_base[b] = static_cast<uint32_t>(exact);
        uint64_t c = 0;
        ceil_div(h_totals[b], capacity, c);
        exact += c;
        particles += h_totals[b];
    }
    if (exact > std::numeric_limits<uint32_t>::max())
        return GF_ERR_RANGE;
    uint64_t bound = 0;
    gf_output_chunk_bound(particles, capacity, bins, &bound);
    if (exact > bound)
        return GF_ERR_LOGIC;
    if (h_fills != nullptr) {
        if (exact > fills_cap)
            return GF_ERR_ARGUMENT;
        uint64_t f = 0;
        for (uint32_t b = 0; b < bins; ++b)
            for (uint64_t off = 0; off < h_totals[b]; off += capacity) {
                const uint64_t rem = h_totals[b] - off;
                h_fills[f++] = static_cast<uint32_t>(rem < capacity ? rem : capacity);
            }
    }
    *h_num_out = static_cast<uint32_t>(exact);
    return GF_OK;
}

// graph/DenseBinTable.hpp:80-91
gf_status gf_build_dense_table(const uint32_t* h_bin_base, uint32_t bins, const uint32_t* h_chunk_indices,
                               uint32_t num_out, uint32_t* h_table)
{
    if (h_bin_base == nullptr || h_table == nullptr || (num_out != 0u && h_chunk_indices == nullptr))
        return GF_ERR_ARGUMENT;
    for (uint32_t b = 0; b < bins; ++b)
        h_table[b] = h_bin_base[b];
    for (uint32_t i = 0; i < num_out; ++i)
        h_table[bins + i] = h_chunk_indices[i];
    return GF_OK;
}

// flow/Execution.hpp:113-124
gf_status gf_tile_count(uint32_t fill, uint32_t tile_size, uint32_t* h_out)
{
    if (tile_size == 0u || h_out == nullptr)
        return GF_ERR_ARGUMENT;
    *h_out = fill == 0u ? 0u : static_cast<uint32_t>((static_cast<uint64_t>(fill) + tile_size - 1u) / tile_size);
    return GF_OK;
}

// flow/Execution.hpp:2377-2389
gf_status gf_flatten_tiles(const uint32_t* h_chunk_index, const uint32_t* h_fills, uint32_t n_chunks,
                           uint32_t tile_size, gf_tile* h_tiles, uint32_t cap, uint32_t* h_n_tiles)
{
    if (tile_size == 0u || h_n_tiles == nullptr || (n_chunks != 0u && (h_chunk_index == nullptr || h_fills == nullptr)))
        return GF_ERR_ARGUMENT;
    uint32_t n = 0;
    for (uint32_t c = 0; c < n_chunks; ++c) {
        uint32_t tiles = 0;
        gf_tile_count(h_fills[c], tile_size, &tiles);
        for (uint32_t t = 0; t < tiles; ++t) {
            if (n >= cap || h_tiles == nullptr)
                return GF_ERR_RANGE;
            const uint32_t off = t * tile_size;
            const uint32_t rem = h_fills[c] - off;
            h_tiles[n].chunk_index = h_chunk_index[c];
            h_tiles[n].tile_offset = off;
            h_tiles[n].count = rem < tile_size ? rem : tile_size;
            ++n;
        }
    }
    *h_n_tiles = n;
    return GF_OK;
}

gf_status gf_zipf_cdf(double s, uint32_t k, double* h_cdf)
{
    if (k == 0u || h_cdf == nullptr || !(s >= 0.0))
        return GF_ERR_ARGUMENT;
    double total = 0.0;
    for (uint32_t r = 0; r < k; ++r) {
        total += std::pow(static_cast<double>(r) + 1.0, -s);
        h_cdf[r] = total;
    }
    for (uint32_t r = 0; r < k; ++r)
        h_cdf[r] /= total;
    h_cdf[k - 1] = 1.0;
    return GF_OK;
}

} // extern "C"
