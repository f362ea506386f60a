// Device-side building blocks shared by every graphflow_b200 kernel: the keyed Philox streams,
// exact division by a run-time divisor, relaxed global loads/stores for inter-CTA publication,
// and the bounded spin used by every wait.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "graphflow_b200.h"

#define GF_HD __host__ __device__ __forceinline__
#define GF_D __device__ __forceinline__

namespace gf {

// ---------------------------------------------------------------------------------------------
// Keyed RNG streams.
// Stream key: rng/ParticleRng.hpp:57-94 (packed (id:32, event:16, purpose:16), SplitMix64 mix).
// Philox4x32 (Salmon et al., SC'11) in the form the reference's pinned engine computes it
// (alpaka 3.0.0 Philox4x32x10, rng/ParticleRng.hpp:22,128): one round with the unbumped key,
// then ten rounds after Weyl key bumps; word 0 multiplied by 0xCD9E8D57, word 2 by 0xD2511F53;
// key = {lo, hi} of the stream key; the first block uses counter {1,0,0,0}; words are consumed
// in order 0..3. Checked against tests/unit/test_philox.cpp:145-150.
// ---------------------------------------------------------------------------------------------
GF_HD uint64_t mix64(uint64_t v)
{
    v ^= v >> 30;
    v *= 0xBF58476D1CE4E5B9ull;
    v ^= v >> 27;
    v *= 0x94D049BB133111EBull;
    v ^= v >> 31;
    return v;
}

GF_HD uint64_t stream_key(uint64_t seed_mixed, uint64_t id, uint64_t event, uint32_t purpose)
{
    // seed_mixed = mix64(seed), hoisted by the caller
    uint64_t packed = (id & 0xFFFFFFFFull) | ((event & 0xFFFFull) << 32) | ((uint64_t)(purpose & 0xFFFFu) << 48);
    return mix64(packed ^ seed_mixed);
}

GF_HD uint32_t mulhi32(uint32_t a, uint32_t b)
{
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

struct Philox4 {
    uint32_t v[4];
};

GF_HD Philox4 philox_block(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 11; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t h0 = mulhi32(c0, 0xCD9E8D57u), l0 = c0 * 0xCD9E8D57u;
        uint32_t h1 = mulhi32(c2, 0xD2511F53u), l1 = c2 * 0xD2511F53u;
        uint32_t n0 = h1 ^ c1 ^ k0;
        uint32_t n2 = h0 ^ c3 ^ k1;
        c0 = n0;
        c1 = l1;
        c2 = n2;
        c3 = l0;
    }
    return Philox4{{c0, c1, c2, c3}};
}

// First block (four draws) of the engine of one stream position.
GF_HD Philox4 first_draws(uint64_t key) { return philox_block(1u, 0u, 0u, 0u, (uint32_t)key, (uint32_t)(key >> 32)); }

// Sequential engine for functors that draw more than four values.
struct Engine {
    uint32_t k0, k1, ctr, pos;
    Philox4 w;
    GF_HD explicit Engine(uint64_t key) : k0((uint32_t)key), k1((uint32_t)(key >> 32)), ctr(0u), pos(4u), w{} {}
    GF_HD uint32_t operator()()
    {
        if (pos == 4u) {
            ++ctr;
            w = philox_block(ctr, 0u, 0u, 0u, k0, k1);
            pos = 0u;
        }
        uint32_t r = pos == 0u ? w.v[0] : pos == 1u ? w.v[1] : pos == 2u ? w.v[2] : w.v[3];
        ++pos;
        return r;
    }
};

// One 32-bit draw per real: top 24 bits for float, all 32 bits for double, both in [0, 1).
GF_HD float uniform_f32(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }
GF_HD double uniform_f64(uint32_t x) { return (double)x * 0x1p-32; }

// ---------------------------------------------------------------------------------------------
// Exact q = n / d and r = n % d for 32-bit n and a run-time 32-bit d: q = hi64(M * n) with
// M = ceil(2^64 / d) (Lemire, Kaser, Kurz, "Faster remainder by direct computation", 2019,
// Theorem 1 with N = 32, F = 64). d = 1 is handled separately because M does not fit.
// ---------------------------------------------------------------------------------------------
struct FastDiv {
    uint32_t d;
    uint64_t m;
    GF_HD FastDiv() : d(1u), m(0u) {}
    GF_HD explicit FastDiv(uint32_t div) : d(div), m(div <= 1u ? 0ull : (~0ull) / div + 1ull) {}
    GF_HD uint32_t div(uint32_t n) const
    {
        if (d == 1u)
            return n;
#ifdef __CUDA_ARCH__
        return (uint32_t)__umul64hi(m, (uint64_t)n);
#else
        return (uint32_t)(((unsigned __int128)m * n) >> 64);
#endif
    }
    GF_HD uint32_t mod(uint32_t n) const { return n - div(n) * d; }
};

// ---------------------------------------------------------------------------------------------
// Inter-CTA publication: one 64-bit word carries value and flag together, so relaxed
// device-scope accesses are sufficient.
// ---------------------------------------------------------------------------------------------
GF_D unsigned long long ld_relaxed_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

GF_D void st_relaxed_u64(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

GF_D uint32_t ld_relaxed_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Streaming read of data that no thread of the kernel writes.
template <typename T>
GF_D T ld_stream(const T* p)
{
    return __ldg(p);
}

GF_D uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

GF_D void set_status(uint32_t* status, uint32_t code)
{
    if (status != nullptr)
        atomicCAS(status, 0u, code);
}

// Every wait in this library is bounded: at most kSpinLimit polls (about 50 ms with the
// back-off), and a wait also gives up as soon as the batch's status word reports a failure, so
// one failed tile cannot make the others spin. A wait that gives up records GF_ERR_TIMEOUT.
constexpr uint32_t kSpinLimit = 1u << 20;

// Poll budget of the waits between CTAs (look-back descriptors, chunk claims, the cooperative
// grid barrier): kSpinLimit unless a front end lowers it for a failure test. One copy per
// translation unit (internal linkage); the C ABI's tuning knob "spin_limit" sets the copy of the
// dense partition entry points (gf_capi.cu). Waits on this CTA's own bulk copies keep kSpinLimit:
// they always complete, and a CTA must not leave with a copy into its shared memory in flight.
static __device__ uint32_t g_spin_limit = kSpinLimit;

// ---------------------------------------------------------------------------------------------
// Synthetic key of stream position (id, 0, 0x100 + dist): uniform (the position's first draw),
// Zipf over `bins` ports (inverse CDF of a uniform double; cdf[b] = P(rank <= b)), all in port 0,
// or round robin (key = id).
// ---------------------------------------------------------------------------------------------
GF_HD uint32_t synthetic_key(int dist, uint64_t seed_mixed, uint64_t id, uint32_t bins, const double* cdf)
{
    if (dist == GF_DIST_UNIFORM || dist == GF_DIST_ZIPF) {
        const uint32_t d = first_draws(stream_key(seed_mixed, id, 0u, 0x100u + (uint32_t)dist)).v[0];
        if (dist == GF_DIST_UNIFORM)
            return d;
        const double u = uniform_f64(d);
        uint32_t lo = 0, hi = bins - 1u;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2u;
            if (u < cdf[mid])
                hi = mid;
            else
                lo = mid + 1u;
        }
        return lo;
    }
    if (dist == GF_DIST_ONE_PORT)
        return 0u;
    return (uint32_t)id;
}

// ---------------------------------------------------------------------------------------------
// Built-in classifiers of the kernel-level sweeps and the kernel-axis examples
// (examples/particle_feedback/KernelAxes.hpp:29-42). A result >= bins is invalid.
// ---------------------------------------------------------------------------------------------
struct KeyClassifier {
    int kind;
    uint32_t bins;
    FastDiv fd;
    uint64_t salt;
    GF_HD uint32_t operator()(uint64_t key) const
    {
        switch (kind) {
        case GF_CLS_KEY_MOD:
        case GF_CLS_ID_BALANCED:
            if (key >> 32)
                return (uint32_t)(key % bins);
            return fd.mod((uint32_t)key);
        case GF_CLS_ID_ONEHOT:
            return 0u;
        case GF_CLS_ID_SKEWED:
            return (key & 7u) == 0u ? (uint32_t)(key % bins) : 0u;
        default:
            return bins;
        }
    }
};

// Inverse of mix64: the hash path's classifier recovers the popularity rank of a mixed key.
GF_HD uint64_t unxorshift64(uint64_t y, unsigned s)
{
    uint64_t x = y;
    for (unsigned i = 0; i < 64u / s + 1u; ++i)
        x = y ^ (x >> s);
    return x;
}

GF_HD uint64_t inv_odd64(uint64_t a)
{
    uint64_t x = a;
    for (int i = 0; i < 6; ++i)
        x *= 2u - a * x;
    return x;
}

GF_HD uint64_t unmix64(uint64_t v)
{
    v = unxorshift64(v, 31);
    v *= 0x319642B2D24D8EC3ull; // inverse of 0x94D049BB133111EB mod 2^64
    v = unxorshift64(v, 27);
    v *= 0x96DE1B173F119089ull; // inverse of 0xBF58476D1CE4E5B9 mod 2^64
    v = unxorshift64(v, 30);
    return v;
}

} // namespace gf
