// Device-aware defaults for the chunk capacity C, the live-particle capacity P and the tile width T
// (core/DevicePolicy.hpp:64-129 types, :344-614 makeDevicePolicy), for the fixed pool layout of
// this build (P chunks of C slots each; there is no slot arena). Host-only.
//
// The rules are the reference's, so a caller that leaves C, P or T out gets the values the
// reference would choose on the same device:
//   T  the logical width (128, at least the warp size) rounded down to a warp multiple, capped so a
//      2 T-entry, 16-byte-per-entry hash table fits the shared memory of one block, and by
//      maxThreadsPerBlock; an explicit T is kept if it fits maxThreadsPerBlock.
//   C  waves x SMs x blocks per SM x T, capped by maxChunkCapacity, by maxBlocksPerGrid x T, by the
//      run size (at least one tile) and, for a derived P, by the payload budget (the largest C
//      whose default P fits, found by bisection); rounded down to a multiple of T. An explicit C is
//      kept if it fits maxChunkCapacity and the grid, and an explicit P shrinks the derived C.
//   P  min(N, ratio x C), clamped to the largest P with P x C x slotBytes <= budget (tile-rounded
//      when at least one tile fits); an explicit P is kept and rejected if it does not fit or
//      exceeds N.
//   budget  explicit, or min(global memory / 8, 3 GiB) on a device (16 MiB for a warp-size-one host
//      profile).
// The accelerator ratio P/C is 8 (DevicePolicy.hpp:53) where Flow resolves its configuration;
// direct callers get the reference's default of 2.
#pragma once

#include <algorithm>
#include <cstdint>
#include <limits>
#include <optional>
#include <stdexcept>
#include <string>

namespace graphflow {

struct DeviceProperties {
    std::uint32_t multiProcessorCount = 0u;
    std::uint32_t warpSize = 32u;
    std::uint32_t maxThreadsPerBlock = 1024u;
    std::uint32_t maxBlocksPerGrid = 0x7FFFFFFFu;
    std::uint32_t sharedMemPerBlockBytes = 48u * 1024u;
    std::uint64_t globalMemBytes = 0u;
};

struct DevicePolicyConfig {
    std::uint32_t waves = 1u;
    std::uint32_t targetBlocksPerSm = 4u;
    std::uint32_t logicalTileWidth = 128u;
    std::uint32_t maxChunkCapacity = 8192u;
    std::uint32_t liveParticlesPerChunk = 2u;
    std::uint64_t memoryBudgetBytes = 0u; // 0: derived from the device
    std::uint32_t memoryBudgetDivisor = 8u;
    std::uint64_t hostBudgetBytes = 16ull << 20;
    std::uint64_t acceleratorBudgetCapBytes = 3ull << 30;
    std::uint64_t slotBytes = 24u; // payload bytes of one slot
    static constexpr std::uint32_t kAcceleratorLiveParticlesPerChunk = 8u;
    static constexpr std::uint64_t kHashEntryBytes = 16u;
};

struct DevicePolicyOverrides {
    std::optional<std::uint32_t> chunkCapacity, liveParticles, tileSize;
};

struct DevicePolicy {
    std::uint32_t chunkCapacity = 0u;
    std::uint32_t liveParticles = 0u;
    bool liveParticlesExplicit = false;
    std::uint32_t tileSize = 0u;
    std::uint64_t memoryBudgetBytes = 0u;
    std::string cap; // what bounded C: explicit, wave, maximum, grid, particles or memory
};

namespace policy_detail {

inline std::uint64_t satMul(std::uint64_t a, std::uint64_t b)
{
    return a != 0u && b > std::numeric_limits<std::uint64_t>::max() / a ? std::numeric_limits<std::uint64_t>::max()
                                                                         : a * b;
}

inline std::uint64_t floorTo(std::uint64_t v, std::uint64_t m) { return v / m * m; }

// P x C x slotBytes <= budget, without overflow.
inline bool fits(std::uint64_t live, std::uint64_t chunk, std::uint64_t budget, std::uint64_t slot)
{
    if (live == 0u || chunk == 0u)
        return true;
    if (live > budget / chunk)
        return false;
    return live * chunk <= budget / slot;
}

// Largest P for a given C, rounded down to a tile when at least one tile fits; 0 if none does.
inline std::uint64_t maxLive(std::uint64_t chunk, std::uint64_t budget, std::uint64_t tile, std::uint64_t slot)
{
    if (chunk == 0u)
        return 0u;
    const std::uint64_t perChunk = satMul(chunk, slot);
    std::uint64_t live = budget / perChunk;
    if (tile > 1u && live >= tile)
        live = floorTo(live, tile);
    return live;
}

inline std::uint64_t budgetOf(const DeviceProperties& d, const DevicePolicyConfig& c)
{
    if (c.memoryBudgetBytes != 0u)
        return c.memoryBudgetBytes;
    if (d.warpSize <= 1u)
        return c.hostBudgetBytes;
    const std::uint64_t byMemory = d.globalMemBytes / c.memoryBudgetDivisor;
    return byMemory == 0u ? std::min(c.hostBudgetBytes, c.acceleratorBudgetCapBytes)
                          : std::min(byMemory, c.acceleratorBudgetCapBytes);
}

} // namespace policy_detail

inline DevicePolicy makeDevicePolicy(const DeviceProperties& d, std::uint64_t n, const DevicePolicyOverrides& o = {},
                                     const DevicePolicyConfig& c = {})
{
    using namespace policy_detail;
    auto fail = [](const std::string& what) { throw std::invalid_argument("graphflow device policy rejected: " + what); };
    if (c.waves == 0u || c.targetBlocksPerSm == 0u || c.logicalTileWidth == 0u || c.maxChunkCapacity == 0u ||
        c.liveParticlesPerChunk == 0u || c.memoryBudgetDivisor == 0u || c.hostBudgetBytes == 0u ||
        c.acceleratorBudgetCapBytes == 0u || c.slotBytes == 0u)
        fail("a zero policy setting (every limit and factor has to be positive)");
    const std::uint64_t warp = d.warpSize == 0u ? 1u : d.warpSize;
    const std::uint64_t threads = d.maxThreadsPerBlock;
    if (threads == 0u)
        fail("the device properties give zero threads per block");
    if (threads < warp)
        fail("fewer threads per block than one warp holds");
    if (d.maxBlocksPerGrid == 0u)
        fail("the device properties give a zero grid limit");
    if (o.liveParticles && (*o.liveParticles == 0u || *o.liveParticles > n))
        fail("the live-particle count is zero or larger than the run's particles");

    // T
    std::uint64_t tile = 0u;
    if (o.tileSize) {
        if (*o.tileSize == 0u)
            fail("a zero tile size was requested");
        if (*o.tileSize > threads)
            fail("the requested tile size needs more threads than one block may have");
        tile = *o.tileSize;
    } else {
        std::uint64_t t = std::max<std::uint64_t>(floorTo(std::max<std::uint64_t>(c.logicalTileWidth, warp), warp), warp);
        const std::uint64_t bySmem = floorTo(d.sharedMemPerBlockBytes / (2u * DevicePolicyConfig::kHashEntryBytes), warp);
        if (bySmem >= warp)
            t = std::min(t, bySmem);
        tile = std::min(t, floorTo(threads, warp));
    }

    const std::uint64_t budget = budgetOf(d, c);

    // C
    const std::uint64_t grid = satMul(d.maxBlocksPerGrid, tile);
    const std::uint64_t launch = std::min<std::uint64_t>(c.maxChunkCapacity, grid);
    if (!o.chunkCapacity && launch < tile)
        fail("no chunk capacity fits a whole tile under the capacity and grid limits");
    const std::uint64_t sms = d.multiProcessorCount == 0u ? 1u : d.multiProcessorCount;
    const std::uint64_t wave = satMul(satMul(satMul(c.waves, sms), c.targetBlocksPerSm), tile);
    std::uint64_t chunk = 0u;
    std::string cap = "explicit";
    if (o.chunkCapacity) {
        if (*o.chunkCapacity == 0u)
            fail("a zero chunk capacity was requested");
        if (*o.chunkCapacity > c.maxChunkCapacity)
            fail("the requested chunk capacity is above the limit of " + std::to_string(c.maxChunkCapacity) + " slots");
        if (*o.chunkCapacity > grid)
            fail("one chunk of the requested capacity would need a grid larger than the device allows");
        chunk = *o.chunkCapacity;
    } else {
        std::uint64_t v = std::min(wave, launch);
        cap = wave <= launch ? "wave" : (c.maxChunkCapacity <= grid ? "maximum" : "grid");
        const std::uint64_t run = std::max<std::uint64_t>(n, tile);
        if (v > run) {
            v = run;
            cap = "particles";
        }
        std::uint64_t byBudget = v;
        if (o.liveParticles) {
            byBudget = budget / satMul(*o.liveParticles, c.slotBytes);
        } else {
            // largest C in [0, v] whose default P = min(N, ratio C) fits the budget
            std::uint64_t lo = 0u, hi = v;
            while (lo < hi) {
                const std::uint64_t mid = lo + (hi - lo + 1u) / 2u;
                if (fits(std::min(n, satMul(c.liveParticlesPerChunk, mid)), mid, budget, c.slotBytes))
                    lo = mid;
                else
                    hi = mid - 1u;
            }
            byBudget = lo;
        }
        if (byBudget < v) {
            v = byBudget;
            cap = "memory";
        }
        v = floorTo(v, tile);
        if (v < tile)
            fail("the memory budget is smaller than one tile of payload");
        chunk = v;
    }

    // P
    const bool liveExplicit = o.liveParticles.has_value();
    std::uint64_t live = 0u;
    if (liveExplicit)
        live = *o.liveParticles;
    else if (n != 0u)
        live = std::min<std::uint64_t>({n, satMul(c.liveParticlesPerChunk, chunk), std::numeric_limits<std::uint32_t>::max()});
    if (live != 0u) {
        std::uint64_t most = maxLive(chunk, budget, tile, c.slotBytes);
        if (most == 0u && !o.chunkCapacity) {
            const std::uint64_t shrunk = floorTo(std::min<std::uint64_t>(chunk, budget / c.slotBytes), tile);
            if (shrunk < tile)
                fail("the memory budget is smaller than one tile of payload");
            chunk = shrunk;
            cap = "memory";
            most = maxLive(chunk, budget, tile, c.slotBytes);
        }
        if (most == 0u)
            fail("the memory budget has no room for a single live particle");
        if (liveExplicit && live > most)
            fail(std::to_string(live) + " live particles at " + std::to_string(chunk) + " slots per chunk do not fit " +
                 std::to_string(budget) + " budget bytes; at most " + std::to_string(most) + " do");
        if (!liveExplicit && live > most) {
            live = most;
            cap = "memory";
        }
    }
    if (!fits(live, chunk, budget, c.slotBytes))
        fail("the live particles at this chunk capacity need more memory than the budget");

    DevicePolicy p;
    p.chunkCapacity = static_cast<std::uint32_t>(chunk);
    p.liveParticles = static_cast<std::uint32_t>(live);
    p.liveParticlesExplicit = liveExplicit;
    p.tileSize = static_cast<std::uint32_t>(tile);
    p.memoryBudgetBytes = budget;
    p.cap = cap;
    return p;
}

} // namespace graphflow
