/* graphFlow-B200 oracle: CPU restatement of the reference hot path. TEST INFRASTRUCTURE ONLY.
 *
 * Only the tests, the smoke check and the CPU-baseline legs of the benchmark use this file, as
 * the checker or as the timed CPU restatement. The product library never links it.
 * Each function names the reference file:line (inside the graphFlow project) that it restates.
 */
#include "gf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------------------------ */
/* keyed RNG                                                                                   */
/* ------------------------------------------------------------------------------------------ */

/* SplitMix64 finalizer: rng/ParticleRng.hpp:69-77 */
uint64_t gfo_mix64(uint64_t v)
{
    v ^= v >> 30;
    v *= 0xBF58476D1CE4E5B9ull;
    v ^= v >> 27;
    v *= 0x94D049BB133111EBull;
    v ^= v >> 31;
    return v;
}

static uint64_t inv_odd64(uint64_t a)
{
    /* Newton iteration for the inverse of an odd number modulo 2^64. */
    uint64_t x = a;
    for (int i = 0; i < 6; ++i)
        x *= 2u - a * x;
    return x;
}

static uint64_t unxorshift(uint64_t y, unsigned s)
{
    uint64_t x = y;
    for (unsigned i = 0; i < 64u / s + 1u; ++i)
        x = y ^ (x >> s);
    return x;
}

/* Inverse of gfo_mix64 (every step of the finalizer is a bijection). */
uint64_t gfo_unmix64(uint64_t v)
{
    v = unxorshift(v, 31);
    v *= inv_odd64(0x94D049BB133111EBull);
    v = unxorshift(v, 27);
    v *= inv_odd64(0xBF58476D1CE4E5B9ull);
    v = unxorshift(v, 30);
    return v;
}

/* packed position + key: rng/ParticleRng.hpp:57-61 and :86-94 */
uint64_t gfo_stream_key(uint64_t seed, uint64_t id, uint64_t event, uint32_t purpose)
{
    uint64_t packed = (id & 0xFFFFFFFFull) | ((event & 0xFFFFull) << 32) | ((uint64_t)(purpose & 0xFFFFu) << 48);
    return gfo_mix64(packed ^ gfo_mix64(seed));
}

/* Philox4x32 block function (Salmon et al., SC'11) in the form the reference's pinned engine
 * computes it: one round with the unbumped key, then ten rounds each after a Weyl key bump.
 * Word 0 is multiplied by 0xCD9E8D57 and word 2 by 0xD2511F53. The layout (key = {lo, hi} of the
 * 64-bit stream key, counter starts at {0,0,0,0} and is incremented before the first block,
 * output words in order 0..3) reproduces every literal of tests/unit/test_philox.cpp:145-150. */
static void philox_round(uint32_t c[4], const uint32_t k[2])
{
    uint64_t p0 = (uint64_t)c[0] * 0xCD9E8D57u;
    uint64_t p1 = (uint64_t)c[2] * 0xD2511F53u;
    uint32_t h0 = (uint32_t)(p0 >> 32), l0 = (uint32_t)p0;
    uint32_t h1 = (uint32_t)(p1 >> 32), l1 = (uint32_t)p1;
    uint32_t n0 = h1 ^ c[1] ^ k[0];
    uint32_t n2 = h0 ^ c[3] ^ k[1];
    c[0] = n0;
    c[1] = l1;
    c[2] = n2;
    c[3] = l0;
}

void gfo_philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k[2] = {key[0], key[1]};
    philox_round(c, k);
    for (int r = 0; r < 10; ++r) {
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
        philox_round(c, k);
    }
    memcpy(out, c, sizeof(c));
}

void gfo_engine_init(gfo_engine* e, uint64_t key)
{
    e->key[0] = (uint32_t)key;
    e->key[1] = (uint32_t)(key >> 32);
    memset(e->ctr, 0, sizeof(e->ctr));
    memset(e->out, 0, sizeof(e->out));
    e->pos = 4u;
}

uint32_t gfo_engine_next(gfo_engine* e)
{
    if (e->pos == 4u) {
        /* 128-bit counter increment */
        for (int w = 0; w < 4; ++w)
            if (++e->ctr[w] != 0u)
                break;
        gfo_philox_block(e->ctr, e->key, e->out);
        e->pos = 0u;
    }
    return e->out[e->pos++];
}

uint32_t gfo_draw(uint64_t seed, uint64_t id, uint64_t event, uint32_t purpose)
{
    gfo_engine e;
    gfo_engine_init(&e, gfo_stream_key(seed, id, event, purpose));
    return gfo_engine_next(&e);
}

void gfo_draws(uint64_t seed, uint64_t id, uint64_t event, uint32_t purpose, uint32_t* out, uint32_t n)
{
    gfo_engine e;
    gfo_engine_init(&e, gfo_stream_key(seed, id, event, purpose));
    for (uint32_t i = 0; i < n; ++i)
        out[i] = gfo_engine_next(&e);
}

/* Word-to-real conversion. The reference draws reals through alpaka's UniformReal, which no
 * reference test pins to a literal; this build uses one 32-bit draw per real: the top 24 bits
 * for float and all 32 bits for double, both in [0, 1). */
float gfo_uniform_f32(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }
double gfo_uniform_f64(uint32_t x) { return (double)x * 0x1p-32; }

/* ------------------------------------------------------------------------------------------ */
/* reservation and exact plan                                                                  */
/* ------------------------------------------------------------------------------------------ */

/* core/Reservation.hpp:15-20 */
int gfo_ceil_div(uint64_t num, uint64_t den, uint64_t* out)
{
    if (den == 0u)
        return GFO_INVALID;
    *out = num / den + (num % den != 0u ? 1u : 0u);
    return GFO_OK;
}

/* core/Reservation.hpp:35-50: R = min(n, ceil(n/C) + min(B, n) - 1) */
int gfo_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint64_t* out)
{
    if (n == 0u) {
        *out = 0u;
        return GFO_OK;
    }
    if (capacity == 0u || max_bins == 0u)
        return GFO_INVALID;
    uint64_t per_chunk;
    gfo_ceil_div(n, capacity, &per_chunk);
    uint64_t bins = max_bins < n ? max_bins : n;
    if (per_chunk > UINT64_MAX - bins + 1u)
        return GFO_OVERFLOW;
    uint64_t bound = per_chunk + bins - 1u;
    *out = bound < n ? bound : n;
    return GFO_OK;
}

/* core/Reservation.hpp:61-71 */
int gfo_checked_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint32_t* out)
{
    uint64_t b;
    int rc = gfo_output_chunk_bound(n, capacity, max_bins, &b);
    if (rc != GFO_OK)
        return rc;
    if (b > UINT32_MAX)
        return GFO_OVERFLOW;
    *out = (uint32_t)b;
    return GFO_OK;
}

/* graph/DenseBinTable.hpp:39-77: binBase = exclusive scan of ceil(total_b / C); fills per chunk */
int gfo_plan_dense(const uint32_t* totals, uint64_t bins, uint32_t capacity, uint32_t* bin_base,
                   uint32_t* fills, uint64_t fills_cap, uint32_t* num_out)
{
    if (bins == 0u || capacity == 0u)
        return GFO_INVALID;
    uint64_t exact = 0u, particles = 0u;
    for (uint64_t b = 0; b < bins; ++b) {
        bin_base[b] = (uint32_t)exact;
        exact += totals[b] / capacity + (totals[b] % capacity != 0u);
        particles += totals[b];
    }
    if (exact > UINT32_MAX)
        return GFO_OVERFLOW;
    uint64_t bound;
    gfo_output_chunk_bound(particles, capacity, bins, &bound);
    if (exact > bound)
        return GFO_LOGIC;
    if (fills != NULL) {
        if (exact > fills_cap)
            return GFO_INVALID;
        uint64_t f = 0;
        for (uint64_t b = 0; b < bins; ++b)
            for (uint32_t off = 0; off < totals[b]; off += capacity) {
                uint32_t rem = totals[b] - off;
                fills[f++] = rem < capacity ? rem : capacity;
                if (off > UINT32_MAX - capacity)
                    break;
            }
    }
    *num_out = (uint32_t)exact;
    return GFO_OK;
}

/* ------------------------------------------------------------------------------------------ */
/* tiles                                                                                       */
/* ------------------------------------------------------------------------------------------ */

/* flow/Execution.hpp:113-124 */
int gfo_tile_count(uint32_t fill, uint32_t tile_size, uint32_t* out)
{
    if (tile_size == 0u)
        return GFO_INVALID;
    *out = fill == 0u ? 0u : (uint32_t)(((uint64_t)fill + tile_size - 1u) / tile_size);
    return GFO_OK;
}

/* flow/Execution.hpp:2377-2389: one descriptor per <= T slice of every chunk, in chunk order */
int64_t gfo_flatten_tiles(const uint32_t* chunk_index, const uint32_t* fills, uint32_t n_chunks,
                          uint32_t tile_size, gfo_tile* out, uint64_t cap)
{
    if (tile_size == 0u)
        return -GFO_INVALID;
    uint64_t n = 0;
    for (uint32_t c = 0; c < n_chunks; ++c) {
        uint32_t tiles;
        gfo_tile_count(fills[c], tile_size, &tiles);
        for (uint32_t t = 0; t < tiles; ++t) {
            if (n >= cap)
                return -GFO_OVERFLOW;
            uint32_t off = t * tile_size;
            uint32_t rem = fills[c] - off;
            out[n].chunk_index = chunk_index[c];
            out[n].tile_offset = off;
            out[n].count = rem < tile_size ? rem : tile_size;
            ++n;
        }
    }
    return (int64_t)n;
}

/* ------------------------------------------------------------------------------------------ */
/* classifiers                                                                                 */
/* ------------------------------------------------------------------------------------------ */

/* Returns a bin, or a value >= bins for an out-of-range result (the reference's status slot). */
uint32_t gfo_classify(int cls, uint64_t key, uint32_t bins, uint64_t salt)
{
    switch (cls) {
    case GFO_CLS_KEY_MOD:
        return (uint32_t)(key % bins);
    case GFO_CLS_ID_BALANCED: /* examples/particle_feedback/KernelAxes.hpp:29-31 */
        return (uint32_t)(key % bins);
    case GFO_CLS_ID_ONEHOT: /* KernelAxes.hpp:34-35 */
        return 0u;
    case GFO_CLS_ID_SKEWED: /* KernelAxes.hpp:38-41 */
        return key % 8u == 0u ? (uint32_t)(key % bins) : 0u;
    case GFO_CLS_KEY_UNMIX: {
        uint64_t r = gfo_unmix64(key) ^ salt;
        return r < bins ? (uint32_t)r : bins;
    }
    default:
        return bins;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* stable partition                                                                            */
/* ------------------------------------------------------------------------------------------ */

static int clamp_threads(int threads)
{
#ifdef _OPENMP
    if (threads <= 0)
        threads = omp_get_max_threads();
#else
    threads = 1;
#endif
    return threads < 1 ? 1 : threads;
}

static int partition_stable(const void* keys, int wide, uint64_t n, uint32_t bins, int cls, uint64_t salt,
                            uint32_t* counts, uint32_t* order, int threads)
{
    threads = clamp_threads(threads);
    if (bins == 0u)
        return GFO_INVALID;
    uint32_t* hist = (uint32_t*)calloc((size_t)threads * bins, sizeof(uint32_t));
    if (!hist)
        return GFO_OVERFLOW;
    int bad = 0;
#pragma omp parallel num_threads(threads) reduction(| : bad)
    {
        int t = 0, nt = 1;
#ifdef _OPENMP
        t = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        uint64_t lo = n * (uint64_t)t / (uint64_t)nt, hi = n * (uint64_t)(t + 1) / (uint64_t)nt;
        uint32_t* h = hist + (size_t)t * bins;
        for (uint64_t i = lo; i < hi; ++i) {
            uint64_t key = wide ? ((const uint64_t*)keys)[i] : ((const uint32_t*)keys)[i];
            uint32_t b = gfo_classify(cls, key, bins, salt);
            if (b >= bins) {
                bad = 1;
                continue;
            }
            h[b]++;
        }
    }
    if (bad) {
        free(hist);
        return GFO_INVALID;
    }
    /* offsets: port-major, then thread order (thread ranges are contiguous => stable) */
    uint64_t run = 0;
    for (uint32_t b = 0; b < bins; ++b) {
        uint64_t total = 0;
        for (int t = 0; t < threads; ++t) {
            uint32_t c = hist[(size_t)t * bins + b];
            hist[(size_t)t * bins + b] = (uint32_t)(run + total);
            total += c;
        }
        counts[b] = (uint32_t)total;
        run += total;
    }
    if (order != NULL) {
#pragma omp parallel num_threads(threads)
        {
            int t = 0, nt = 1;
#ifdef _OPENMP
            t = omp_get_thread_num();
            nt = omp_get_num_threads();
#endif
            uint64_t lo = n * (uint64_t)t / (uint64_t)nt, hi = n * (uint64_t)(t + 1) / (uint64_t)nt;
            uint32_t* h = hist + (size_t)t * bins;
            for (uint64_t i = lo; i < hi; ++i) {
                uint64_t key = wide ? ((const uint64_t*)keys)[i] : ((const uint32_t*)keys)[i];
                uint32_t b = gfo_classify(cls, key, bins, salt);
                order[h[b]++] = (uint32_t)i;
            }
        }
    }
    free(hist);
    return GFO_OK;
}

int gfo_partition_stable_u32(const uint32_t* keys, uint64_t n, uint32_t bins, int cls, uint32_t* counts,
                             uint32_t* order, int threads)
{
    return partition_stable(keys, 0, n, bins, cls, 0u, counts, order, threads);
}

int gfo_partition_stable_u64(const uint64_t* keys, uint64_t n, uint32_t bins, int cls, uint64_t salt,
                             uint32_t* counts, uint32_t* order, int threads)
{
    return partition_stable(keys, 1, n, bins, cls, salt, counts, order, threads);
}

/* Reference-structured pool path: classify (ClassifyKernel.hpp:57-91), plan
 * (Execution.hpp:2520-2590 with DenseBinTable.hpp:39-91), scatter with the per-tile reservation
 * and shared cursor (ScatterKernel.hpp:279-366), output descriptors (Execution.hpp:2558-2581). */
int gfo_partition_pool_u32(const uint32_t* pool_in, uint32_t* pool_out, uint32_t capacity, const gfo_tile* tiles,
                           uint64_t n_tiles, uint32_t bins, int cls, uint32_t* bin_ids, uint32_t* counts,
                           const uint32_t* free_chunks, uint64_t n_free, uint32_t* table, gfo_out_desc* outs,
                           uint32_t* n_outs, int threads)
{
    threads = clamp_threads(threads);
    if (bins == 0u || capacity == 0u)
        return GFO_INVALID;
    memset(counts, 0, sizeof(uint32_t) * bins);
    int bad = 0;
    uint64_t particles = 0;
#pragma omp parallel num_threads(threads) reduction(| : bad) reduction(+ : particles)
    {
        uint32_t* local = (uint32_t*)calloc(bins, sizeof(uint32_t));
#pragma omp for schedule(static)
        for (int64_t t = 0; t < (int64_t)n_tiles; ++t) {
            uint64_t base = (uint64_t)tiles[t].chunk_index * capacity + tiles[t].tile_offset;
            for (uint32_t i = 0; i < tiles[t].count; ++i) {
                uint32_t b = gfo_classify(cls, pool_in[base + i], bins, 0u);
                if (b >= bins) {
                    bad = 1;
                    continue;
                }
                bin_ids[base + i] = b;
                local[b]++;
            }
            particles += tiles[t].count;
        }
        for (uint32_t b = 0; b < bins; ++b)
            if (local[b])
#pragma omp atomic
                counts[b] += local[b];
        free(local);
    }
    if (bad)
        return GFO_INVALID;
    uint32_t* fills = (uint32_t*)malloc(sizeof(uint32_t) * (n_free + 1));
    uint32_t R = 0;
    int rc = gfo_plan_dense(counts, bins, capacity, table, fills, n_free, &R);
    if (rc != GFO_OK) {
        free(fills);
        return rc;
    }
    if (R > n_free) {
        free(fills);
        return GFO_OVERFLOW;
    }
    uint32_t f = 0;
    for (uint32_t b = 0; b < bins; ++b) {
        uint32_t nb = counts[b] / capacity + (counts[b] % capacity != 0u);
        for (uint32_t k = 0; k < nb; ++k, ++f) {
            table[bins + f] = free_chunks[f];
            outs[f].chunk_index = free_chunks[f];
            outs[f].fill = fills[f];
            outs[f].bin = b;
        }
    }
    *n_outs = R;
    free(fills);
    uint32_t* next = (uint32_t*)calloc(bins, sizeof(uint32_t));
#pragma omp parallel num_threads(threads)
    {
        uint32_t* cnt = (uint32_t*)malloc(sizeof(uint32_t) * bins);
        uint32_t* cur = (uint32_t*)malloc(sizeof(uint32_t) * bins);
#pragma omp for schedule(static)
        for (int64_t t = 0; t < (int64_t)n_tiles; ++t) {
            uint64_t base = (uint64_t)tiles[t].chunk_index * capacity + tiles[t].tile_offset;
            uint32_t cnt_n = tiles[t].count;
            memset(cnt, 0, sizeof(uint32_t) * bins);
            for (uint32_t i = 0; i < cnt_n; ++i)
                cnt[bin_ids[base + i]]++;
            for (uint32_t i = 0; i < cnt_n; ++i) {
                uint32_t b = bin_ids[base + i];
                if (cnt[b] != 0u) {
                    cur[b] = __atomic_fetch_add(&next[b], cnt[b], __ATOMIC_RELAXED);
                    cnt[b] = 0u;
                }
            }
            for (uint32_t i = 0; i < cnt_n; ++i) {
                uint32_t b = bin_ids[base + i];
                uint32_t j = cur[b]++;
                uint32_t chunk = table[bins + table[b] + j / capacity];
                pool_out[(uint64_t)chunk * capacity + j % capacity] = pool_in[base + i];
            }
        }
        free(cnt);
        free(cur);
    }
    int ok = 1;
    for (uint32_t b = 0; b < bins; ++b)
        ok &= next[b] == counts[b]; /* finalise: Execution.hpp:2715-2725 */
    free(next);
    (void)particles;
    return ok ? GFO_OK : GFO_LOGIC;
}

/* ------------------------------------------------------------------------------------------ */
/* synthetic key distributions                                                                 */
/* ------------------------------------------------------------------------------------------ */

uint32_t gfo_dist_purpose(int dist) { return 0x100u + (uint32_t)dist; }

void gfo_zipf_cdf(double s, uint32_t k, double* cdf)
{
    double total = 0.0;
    for (uint32_t r = 0; r < k; ++r) {
        total += pow((double)r + 1.0, -s);
        cdf[r] = total;
    }
    for (uint32_t r = 0; r < k; ++r)
        cdf[r] /= total;
    cdf[k - 1] = 1.0;
}

/* smallest r with u < cdf[r], u = draw * 2^-32 */
uint32_t gfo_zipf_sample(const double* cdf, uint32_t k, uint32_t draw)
{
    double u = gfo_uniform_f64(draw);
    uint32_t lo = 0, hi = k - 1u;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2u;
        if (u < cdf[mid])
            hi = mid;
        else
            lo = mid + 1u;
    }
    return lo;
}

void gfo_generate_keys_u32(int dist, uint64_t seed, uint64_t first_id, uint64_t n, uint32_t bins, const double* cdf,
                           uint32_t* keys, int threads)
{
    threads = clamp_threads(threads);
    uint32_t purpose = gfo_dist_purpose(dist);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t id = first_id + (uint64_t)i;
        uint32_t k;
        switch (dist) {
        case GFO_DIST_UNIFORM:
            k = gfo_draw(seed, id, 0u, purpose);
            break;
        case GFO_DIST_ZIPF:
            k = gfo_zipf_sample(cdf, bins, gfo_draw(seed, id, 0u, purpose));
            break;
        case GFO_DIST_ONE_PORT:
            k = 0u;
            break;
        default:
            k = (uint32_t)id;
            break;
        }
        keys[i] = k;
    }
}

void gfo_generate_records16(uint64_t seed, uint64_t first_id, uint64_t n, const double* cdf, uint32_t k,
                            uint64_t salt, uint64_t* keys, float* weights, uint32_t* tags, int threads)
{
    threads = clamp_threads(threads);
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t id = first_id + (uint64_t)i;
        uint32_t d[2];
        gfo_draws(seed, id, 0u, 0x110u, d, 2u);
        uint32_t r = gfo_zipf_sample(cdf, k, d[0]);
        keys[i] = gfo_mix64((uint64_t)r ^ salt);
        weights[i] = 1.0f - gfo_uniform_f32(d[1]);
        tags[i] = (uint32_t)id;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* particle_feedback scalar model: tests/reference/ScalarModel.hpp:84-133                     */
/* purposes: source 0, filter 2, process A 4, process B 6 (ScalarModel.hpp:32-36)             */
/* ------------------------------------------------------------------------------------------ */

int gfo_particle_scalar(uint64_t seed, uint64_t n, uint32_t max_visits, uint32_t* weights, uint8_t* capped,
                        uint64_t* capped_count, int threads)
{
    threads = clamp_threads(threads);
    uint64_t ncap = 0;
    int overflow = 0;
#pragma omp parallel for num_threads(threads) schedule(static) reduction(+ : ncap) reduction(| : overflow)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t id = (uint64_t)i;
        uint32_t property = gfo_draw(seed, id, 0u, 0u);
        uint32_t weight = 0u, visit = 0u;
        int stage_b = 0; /* filter decision */
        uint8_t is_capped = 0;
        for (;;) {
            uint32_t decision = gfo_draw(seed, id, visit, 2u);
            stage_b = decision >= property;
            uint32_t purpose = stage_b ? 6u : 4u;
            uint32_t inc = stage_b ? 1u : 1000u;
            int survives = gfo_draw(seed, id, visit, purpose) >= 0x80000000u;
            if (!survives)
                break;
            if (visit >= max_visits) {
                is_capped = 1;
                ncap++;
                break;
            }
            if (weight > UINT32_MAX - inc) {
                overflow = 1;
                break;
            }
            weight += inc;
            ++visit;
        }
        weights[i] = weight;
        if (capped)
            capped[i] = is_capped;
    }
    if (capped_count)
        *capped_count = ncap;
    return overflow ? GFO_OVERFLOW : GFO_OK;
}

/* LSD radix sort (4 x 8 bits) then run-length encoding: ParticleTypes.hpp:206-219 */
uint64_t gfo_histogram_u32(uint32_t* values, uint64_t n, uint32_t* row_weight, uint64_t* row_count)
{
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* src = values;
    uint32_t* dst = tmp;
    for (int pass = 0; pass < 4; ++pass) {
        uint64_t cnt[256] = {0};
        int shift = pass * 8;
        for (uint64_t i = 0; i < n; ++i)
            cnt[(src[i] >> shift) & 0xFFu]++;
        uint64_t run = 0;
        for (int d = 0; d < 256; ++d) {
            uint64_t c = cnt[d];
            cnt[d] = run;
            run += c;
        }
        for (uint64_t i = 0; i < n; ++i)
            dst[cnt[(src[i] >> shift) & 0xFFu]++] = src[i];
        uint32_t* s = src;
        src = dst;
        dst = s;
    }
    /* after 4 passes the sorted data is back in `values` */
    free(tmp);
    uint64_t rows = 0;
    for (uint64_t i = 0; i < n;) {
        uint64_t j = i;
        while (j < n && values[j] == values[i])
            ++j;
        if (row_weight)
            row_weight[rows] = values[i];
        if (row_count)
            row_count[rows] = j - i;
        ++rows;
        i = j;
    }
    return rows;
}

/* ------------------------------------------------------------------------------------------ */
/* photon analog transport: tests/reference/ScalarTransport.hpp:87-209                        */
/* purposes: flight 2, scatter 6 (ScalarTransport.hpp:30-32)                                  */
/* ------------------------------------------------------------------------------------------ */

/* Bounded path trace of one id (PhotonFunctors.hpp:201-234): a vertex past the bound sets the
 * truncation flag; ids at or above trace_ids record nothing. */
typedef struct {
    uint64_t ids;
    uint32_t max_vertices;
    gfo_trace_vertex* vertices;
    uint32_t* counts;
    uint32_t* truncated;
} photon_trace;

static void trace_record(const photon_trace* tr, uint64_t id, uint32_t kind, uint32_t sc, double x, double y,
                         double z, double ux, double uy, double uz)
{
    if (id >= tr->ids)
        return;
    uint32_t index = tr->counts[id];
    if (index >= tr->max_vertices) {
        tr->truncated[id] = 1u;
        return;
    }
    gfo_trace_vertex v = {kind, sc, x, y, z, ux, uy, uz};
    tr->vertices[id * tr->max_vertices + index] = v;
    tr->counts[id] = index + 1u;
}

static int photon_analog_run(uint64_t seed, uint64_t n, double thickness, double sigma_s, double sigma_a,
                             int isotropic, uint32_t max_scatters, gfo_photon_terminal* out, const photon_trace* tr,
                             int threads)
{
    if (!(thickness > 0.0) || !isfinite(thickness) || sigma_s < 0.0 || sigma_a < 0.0)
        return GFO_INVALID;
    threads = clamp_threads(threads);
    double total = sigma_s + sigma_a;
    int bad = 0;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1024) reduction(| : bad)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t id = (uint64_t)i;
        double x = 0, y = 0, z = 0, ux = 0, uy = 0, uz = 1;
        uint32_t sc = 0;
        gfo_photon_terminal t;
        trace_record(tr, id, 0u, 0u, x, y, z, ux, uy, uz);
        for (;;) {
            int reach = 0;
            double fd = 0.0;
            uint32_t fe = 3u;
            if (uz > 0.0) {
                reach = 1;
                fd = (thickness - z) / uz;
                fe = 1u;
            } else if (uz < 0.0) {
                reach = 1;
                fd = -z / uz;
                fe = 2u;
            }
            if (total == 0.0) {
                if (!reach) {
                    bad = 1;
                    t.event = 3u;
                    break;
                }
                x += fd * ux;
                y += fd * uy;
                z = fe == 1u ? thickness : 0.0;
                t.event = fe;
                break;
            }
            uint32_t d[2];
            gfo_draws(seed, id, sc, 2u, d, 2u);
            double flight = 1.0 - gfo_uniform_f64(d[0]);
            double kind = gfo_uniform_f64(d[1]);
            double s = -log(flight) / total;
            if (reach && fd <= s) {
                x += fd * ux;
                y += fd * uy;
                z = fe == 1u ? thickness : 0.0;
                t.event = fe;
                break;
            }
            int scatters = kind < sigma_s / total;
            x += s * ux;
            y += s * uy;
            z += s * uz;
            if (!scatters) {
                t.event = 3u;
                break;
            }
            if (sc >= max_scatters) {
                t.event = 4u;
                break;
            }
            if (isotropic) {
                uint32_t e[2];
                gfo_draws(seed, id, sc, 6u, e, 2u);
                double mu = 2.0 * gfo_uniform_f64(e[0]) - 1.0;
                double phi = 2.0 * M_PI * gfo_uniform_f64(e[1]);
                double tr = sqrt(fmax(0.0, 1.0 - mu * mu));
                ux = tr * cos(phi);
                uy = tr * sin(phi);
                uz = mu;
            }
            trace_record(tr, id, 1u, sc + 1u, x, y, z, ux, uy, uz);
            ++sc;
        }
        trace_record(tr, id, t.event + 1u, sc, x, y, z, ux, uy, uz);
        t.scatter_count = sc;
        t.x = x;
        t.y = y;
        t.z = z;
        t.ux = ux;
        t.uy = uy;
        t.uz = uz;
        out[i] = t;
    }
    return bad ? GFO_INVALID : GFO_OK;
}

int gfo_photon_analog(uint64_t seed, uint64_t n, double thickness, double sigma_s, double sigma_a, int isotropic,
                      uint32_t max_scatters, gfo_photon_terminal* out, int threads)
{
    photon_trace none = {0u, 0u, NULL, NULL, NULL};
    return photon_analog_run(seed, n, thickness, sigma_s, sigma_a, isotropic, max_scatters, out, &none, threads);
}

int gfo_photon_analog_traced(uint64_t seed, uint64_t n, double thickness, double sigma_s, double sigma_a,
                             int isotropic, uint32_t max_scatters, gfo_photon_terminal* out, uint32_t trace_photons,
                             uint32_t trace_vertices, gfo_trace_vertex* vertices, uint32_t* counts,
                             uint32_t* truncated, int threads)
{
    photon_trace tr = {trace_photons < n ? trace_photons : n, trace_vertices, vertices, counts, truncated};
    for (uint64_t id = 0; id < tr.ids; ++id)
        counts[id] = truncated[id] = 0u;
    return photon_analog_run(seed, n, thickness, sigma_s, sigma_a, isotropic, max_scatters, out, &tr, threads);
}

/* ------------------------------------------------------------------------------------------ */
/* weighted slab photon model (Henyey-Greenstein, implicit capture, Russian roulette)          */
/* Stages and stream purposes follow the reference topology (PhotonScattering.hpp:84-102):     */
/* propose flight = node 1 (purpose 2: flight draw, roulette draw), scatter = node 3          */
/* (purpose 6: HG cosine draw, azimuth draw). HG sampling and the direction update are the     */
/* published MCML forms (Wang, Jacques, Zheng 1995).                                           */
/* ------------------------------------------------------------------------------------------ */

static double hg_cos(double g, double xi)
{
    if (g == 0.0)
        return 2.0 * xi - 1.0;
    double t = (1.0 - g * g) / (1.0 - g + 2.0 * g * xi);
    double c = (1.0 + g * g - t * t) / (2.0 * g);
    return c < -1.0 ? -1.0 : (c > 1.0 ? 1.0 : c);
}

int gfo_photon_hg(uint64_t seed, uint64_t first_id, uint64_t n, const gfo_hg_params* p, gfo_hg_terminal* out,
                  double* refl_hist, double* trans_hist, uint64_t* event_counts, int threads)
{
    threads = clamp_threads(threads);
    double L = p->thickness, mt = p->mu_a + p->mu_s, albedo = p->mu_s / (p->mu_a + p->mu_s);
    uint32_t nb = p->hist_bins;
    if (!(L > 0.0) || !(mt > 0.0) || nb == 0u)
        return GFO_INVALID;
    if (refl_hist)
        memset(refl_hist, 0, sizeof(double) * nb);
    if (trans_hist)
        memset(trans_hist, 0, sizeof(double) * nb);
    uint64_t ev[5] = {0, 0, 0, 0, 0};
    /* per-thread partial histograms over static id ranges, summed in thread order afterwards,
     * so the FP64 sums are reproducible for a fixed thread count */
    double* partial = (double*)calloc((size_t)threads * 2u * nb, sizeof(double));
    uint64_t* pev = (uint64_t*)calloc((size_t)threads * 5u, sizeof(uint64_t));
#pragma omp parallel num_threads(threads)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* rh = partial + (size_t)tid * 2u * nb;
        double* th = rh + nb;
        uint64_t* lev = pev + (size_t)tid * 5u;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            uint64_t id = first_id + (uint64_t)i;
            double x = 0, y = 0, z = 0, ux = 0, uy = 0, uz = 1, w = 1.0;
            uint32_t sc = 0, event;
            for (;;) {
                uint32_t d[2];
                gfo_draws(seed, id, sc, 2u, d, 2u);
                double s = -log(1.0 - gfo_uniform_f64(d[0])) / mt;
                int reach = 0;
                double fd = 0.0;
                uint32_t fe = 3u;
                if (uz > 0.0) {
                    reach = 1;
                    fd = (L - z) / uz;
                    fe = 1u;
                } else if (uz < 0.0) {
                    reach = 1;
                    fd = -z / uz;
                    fe = 2u;
                }
                if (reach && fd <= s) {
                    x += fd * ux;
                    y += fd * uy;
                    z = fe == 1u ? L : 0.0;
                    event = fe;
                    break;
                }
                x += s * ux;
                y += s * uy;
                z += s * uz;
                w *= albedo;
                if (w < p->roulette_threshold) {
                    if (gfo_uniform_f64(d[1]) < p->roulette_survival)
                        w /= p->roulette_survival;
                    else {
                        event = 3u;
                        break;
                    }
                }
                if (sc >= p->max_scatters) {
                    event = 4u;
                    break;
                }
                uint32_t e[2];
                gfo_draws(seed, id, sc, 6u, e, 2u);
                double ct = hg_cos(p->g, gfo_uniform_f64(e[0]));
                double phi = 2.0 * M_PI * gfo_uniform_f64(e[1]);
                double st = sqrt(fmax(0.0, 1.0 - ct * ct));
                double cp = cos(phi), sp = sin(phi);
                if (fabs(uz) > 1.0 - 1e-12) {
                    ux = st * cp;
                    uy = st * sp;
                    uz = uz >= 0.0 ? ct : -ct;
                } else {
                    double tmp = sqrt(1.0 - uz * uz);
                    double nx = st * (ux * uz * cp - uy * sp) / tmp + ux * ct;
                    double ny = st * (uy * uz * cp + ux * sp) / tmp + uy * ct;
                    double nz = -st * cp * tmp + uz * ct;
                    ux = nx;
                    uy = ny;
                    uz = nz;
                }
                ++sc;
            }
            double c = fabs(uz);
            uint32_t bin = (uint32_t)(c * nb);
            if (bin >= nb)
                bin = nb - 1u;
            if (event == 1u)
                th[bin] += w;
            else if (event == 2u)
                rh[bin] += w;
            lev[event]++;
            if (out) {
                out[i].event = event;
                out[i].scatter_count = sc;
                out[i].weight = w;
                out[i].cos_exit = c;
            }
        }
    }
    for (int t = 0; t < threads; ++t) {
        for (uint32_t b = 0; b < nb; ++b) {
            if (refl_hist)
                refl_hist[b] += partial[(size_t)t * 2u * nb + b];
            if (trans_hist)
                trans_hist[b] += partial[(size_t)t * 2u * nb + nb + b];
        }
        for (int k = 0; k < 5; ++k)
            ev[k] += pev[(size_t)t * 5u + k];
    }
    free(partial);
    free(pev);
    if (event_counts)
        memcpy(event_counts, ev, sizeof(ev));
    return GFO_OK;
}
