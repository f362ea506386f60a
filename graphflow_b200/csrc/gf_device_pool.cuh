// Device-resident chunk pool: the free list, the per-chunk ledger and the reservation credits of
// the host pool (core/ChunkPool.hpp:88-190, core/ChunkLedger.hpp:33-150, the credit loop of
// sched/GraphRunner.hpp:1014-1037) kept in device memory, so that a flow whose nodes all run on
// the device (one stream, no host round trip between nodes) takes and returns chunks in stream
// order.
//
// Layout (one device allocation of gf_device_pool_bytes(S)): a 64-byte header, ids[S], state[S].
//   free list  ids[base .. S) are the free chunks and ids[base] is handed out next. A fresh pool
//              holds 0, 1, ..., S-1 in that order, so consecutive acquisitions return chunks 0, 1,
//              2, ... as the host pool does (its free vector is filled S-1 .. 0 and popped from the
//              back); a release pushes in front of base, so the chunk released last is handed out
//              first (the host pool's push_back / back order).
//   ledger     state[c] = generation << 1 | live (a 30-bit generation that wraps). An acquisition
//              finds the live bit clear and sets it; a release finds it set, clears it and
//              advances the generation. A release of a chunk that is not live (released twice, or
//              never acquired) or out of range fails the whole release, changes nothing and
//              records GF_INVALID in the header.
//   credits    a batch reserves its outputChunkBound up front: the reservation pops that many ids
//              (GF_OVERFLOW, and nothing taken, when fewer are free). The batch uses a prefix of
//              them; the settle step after it pushes the unused ones back where they were, so the
//              free list ends exactly as if only the used chunks had been taken (their ledger
//              state returns to free without a generation step), then releases the batch's input
//              chunks.
// Each operation is one single-CTA kernel on the caller's stream (or the same work in block 0 of a
// larger kernel). Operations on one pool must be stream-ordered, like the launches that share a
// fused partition's scratch.
#pragma once

#include "gf_device.cuh"

namespace gf {
namespace { // internal linkage: every translation unit that uses the pool has its own kernels

struct DevicePoolHdr {
    uint32_t num_chunks;         // S
    uint32_t base;               // free chunks are ids[base .. S)
    uint32_t peak_live;          // most chunks out of the pool at once
    uint32_t status;             // GF_OK, or the first failed operation's code
    unsigned long long acquired; // acquisitions over the pool's life (unused reservations excluded)
    unsigned long long released; // releases over the pool's life
    uint32_t pad[8];
};
static_assert(sizeof(DevicePoolHdr) == 64u, "header is 64 bytes");

constexpr int kPoolThreads = 1024;

GF_HD uint64_t device_pool_bytes(uint32_t num_chunks)
{
    return sizeof(DevicePoolHdr) + 8ull * num_chunks;
}

GF_D uint32_t* pool_ids(DevicePoolHdr* h) { return reinterpret_cast<uint32_t*>(h + 1); }
GF_D uint32_t* pool_state(DevicePoolHdr* h) { return pool_ids(h) + h->num_chunks; }

// Records `code` as the pool's failure (first one wins) and in the caller's status word.
GF_D void pool_fail(DevicePoolHdr* h, uint32_t* status, uint32_t code)
{
    atomicCAS(&h->status, 0u, code);
    if (status != nullptr)
        set_status(status, code);
}

__global__ void __launch_bounds__(kPoolThreads) pool_init_kernel(DevicePoolHdr* h, uint32_t S)
{
    uint32_t* ids = reinterpret_cast<uint32_t*>(h + 1);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S; i += gridDim.x * blockDim.x) {
        ids[i] = i;
        ids[S + i] = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        h->num_chunks = S;
        h->base = 0u;
        h->peak_live = 0u;
        h->status = 0u;
        h->acquired = 0ull;
        h->released = 0ull;
    }
}

// Reserves k chunks: pops ids[base .. base + k) into out[0..k) and marks them live. Fewer than k
// free: GF_OVERFLOW, nothing taken, out[] filled with kNoChunk (every kernel that writes through
// a reservation rejects that id).
// The work of one CTA (all of its threads take part); other kernels may run it in their block 0.
GF_D void pool_acquire_block(DevicePoolHdr* h, uint32_t k, uint32_t* out, uint32_t* status)
{
    __shared__ uint32_t s_base, s_ok, s_bad;
    if (threadIdx.x == 0) {
        s_base = h->base;
        s_ok = k <= h->num_chunks - s_base ? 1u : 0u;
        s_bad = 0u;
        if (!s_ok)
            pool_fail(h, status, GF_OVERFLOW);
    }
    __syncthreads();
    uint32_t* ids = pool_ids(h);
    uint32_t* state = pool_state(h);
    const uint32_t base = s_base;
    if (!s_ok) {
        for (uint32_t i = threadIdx.x; i < k; i += blockDim.x)
            out[i] = 0xFFFFFFFFu;
        return;
    }
    for (uint32_t i = threadIdx.x; i < k; i += blockDim.x) {
        const uint32_t id = ids[base + i];
        const uint32_t st = id < h->num_chunks ? state[id] : 1u;
        if (st & 1u) // a free-list entry that is live: the pool is corrupted
            s_bad = 1u;
        else
            state[id] = st | 1u;
        out[i] = id;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_bad)
            pool_fail(h, status, GF_INVALID);
        h->base = base + k;
        const uint32_t live = base + k; // chunks out of the pool: every id in front of base
        h->peak_live = live > h->peak_live ? live : h->peak_live;
        h->acquired += k;
    }
}

__global__ void __launch_bounds__(kPoolThreads)
    pool_acquire_kernel(DevicePoolHdr* h, uint32_t k, uint32_t* out, uint32_t* status)
{
    pool_acquire_block(h, k, out, status);
}

// Settles a batch: of its reservation `reserved[0..reserved_n)` the first *d_used (or `used` when
// d_used is null, clamped to reserved_n) were used; the rest go back where they were. Then the
// input chunks in[j * in_stride], j < *d_in_count (or in_count), are released (in_stride 1 for an
// id array, 3 for the chunk_index field of gf_out_desc records). reserved may be null with
// reserved_n = 0, in may be null with a zero count. Any misuse (unused ids no longer just in front
// of base, a released chunk that is out of range, not live, one of the unused reservations or named
// twice) changes nothing and records GF_INVALID.
// The work of one CTA (all of its threads take part); other kernels may run it in their block 0.
GF_D void pool_settle_block(DevicePoolHdr* h, const uint32_t* reserved, uint32_t reserved_n, const uint32_t* d_used,
                            uint32_t used, const uint32_t* in, uint32_t in_stride, const uint32_t* d_in_count,
                            uint32_t in_count, uint32_t* status)
{
    constexpr uint32_t kMark = 0x80000000u; // set only inside this kernel: "released by this call"
    __shared__ uint32_t s_base, s_unused, s_k, s_bad;
    uint32_t* ids = pool_ids(h);
    uint32_t* state = pool_state(h);
    const uint32_t S = h->num_chunks;
    if (threadIdx.x == 0) {
        const uint32_t u = d_used != nullptr ? *d_used : used;
        s_unused = reserved_n - (u < reserved_n ? u : reserved_n);
        s_k = d_in_count != nullptr ? *d_in_count : in_count;
        s_base = h->base;
        s_bad = s_unused > s_base ? 1u : 0u;
    }
    __syncthreads();
    const uint32_t unused = s_unused, k = s_k, base = s_base;
    if (s_bad == 0u) // the unused ids must still sit just in front of base (no pool use in between)
        for (uint32_t j = threadIdx.x; j < unused; j += blockDim.x)
            if (ids[base - unused + j] != reserved[reserved_n - unused + j])
                s_bad = 1u;
    __syncthreads();
    if (s_bad != 0u) {
        if (threadIdx.x == 0)
            pool_fail(h, status, GF_INVALID);
        return;
    }
    // the unused reservations are free again first, so a release that names one of them fails
    for (uint32_t j = threadIdx.x; j < unused; j += blockDim.x)
        atomicAnd(&state[ids[base - unused + j]], ~1u);
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        const uint32_t id = in[(size_t)j * in_stride];
        if (id >= S) {
            s_bad = 1u;
            continue;
        }
        const uint32_t old = atomicOr(&state[id], kMark);
        if ((old & kMark) != 0u || (old & 1u) == 0u) // named twice, or not live
            s_bad = 1u;
    }
    __syncthreads();
    if (s_bad != 0u) { // undo: no mark bit was set before this call, every unused id was live
        for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
            const uint32_t id = in[(size_t)j * in_stride];
            if (id < S)
                atomicAnd(&state[id], ~kMark);
        }
        for (uint32_t j = threadIdx.x; j < unused; j += blockDim.x)
            atomicOr(&state[ids[base - unused + j]], 1u);
        if (threadIdx.x == 0)
            pool_fail(h, status, GF_INVALID);
        return;
    }
    // base chunks are out of the pool, unused + k of them distinct and live here: k <= base - unused.
    // Releases step the generation and are pushed in front (the last one named is handed out first).
    const uint32_t nb = base - unused - k;
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        const uint32_t id = in[(size_t)j * in_stride];
        state[id] = ((state[id] & ~(kMark | 1u)) + 2u) & ~kMark;
        ids[nb + (k - 1u - j)] = id;
    }
    if (threadIdx.x == 0) {
        h->base = nb;
        h->acquired -= unused;
        h->released += k;
    }
}

__global__ void __launch_bounds__(kPoolThreads)
    pool_settle_kernel(DevicePoolHdr* h, const uint32_t* reserved, uint32_t reserved_n, const uint32_t* d_used,
                       uint32_t used, const uint32_t* in, uint32_t in_stride, const uint32_t* d_in_count,
                       uint32_t in_count, uint32_t* status)
{
    pool_settle_block(h, reserved, reserved_n, d_used, used, in, in_stride, d_in_count, in_count, status);
}

} // namespace
} // namespace gf
