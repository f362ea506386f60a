/* graphFlow-B200 oracle: a plain-C CPU restatement of the reference's transform-batch hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Only the tests, the smoke check and the CPU-baseline legs of the
 * benchmark load this library, and only as the checker (or the timed CPU restatement). The
 * product path in graphflow_b200/ never links, loads or calls anything in this directory.
 *
 * Every function cites the reference file:line it restates (paths inside the graphFlow project).
 * The Philox mapping is pinned against the six literals of tests/unit/test_philox.cpp:145-150;
 * the reservation bound and the dense plan against tests/unit/test_reservation.cpp:49-105 and
 * tests/unit/test_dense_bin_table.cpp:18-59.
 */
#ifndef GF_ORACLE_H
#define GF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes (mirror std::invalid_argument / std::overflow_error / std::logic_error) ---- */
enum { GFO_OK = 0, GFO_INVALID = 1, GFO_OVERFLOW = 2, GFO_LOGIC = 3 };

/* ---- keyed RNG (include/graphFlow/rng/ParticleRng.hpp:57-129) ---- */
uint64_t gfo_mix64(uint64_t v);
uint64_t gfo_unmix64(uint64_t v);
uint64_t gfo_stream_key(uint64_t seed, uint64_t id, uint64_t event, uint32_t purpose);

typedef struct {
    uint32_t key[2];
    uint32_t ctr[4];
    uint32_t out[4];
    uint32_t pos;
} gfo_engine;

void gfo_philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void gfo_engine_init(gfo_engine* e, uint64_t key);
uint32_t gfo_engine_next(gfo_engine* e);
/* first u32 draw of the engine at (seed, id, event, purpose) */
uint32_t gfo_draw(uint64_t seed, uint64_t id, uint64_t event, uint32_t purpose);
/* fill out[0..n) with the first n draws of one engine */
void gfo_draws(uint64_t seed, uint64_t id, uint64_t event, uint32_t purpose, uint32_t* out, uint32_t n);
float gfo_uniform_f32(uint32_t x);  /* [0,1) */
double gfo_uniform_f64(uint32_t x); /* [0,1) */

/* ---- reservation and exact plan (core/Reservation.hpp:15-71, graph/DenseBinTable.hpp:39-91) ---- */
int gfo_ceil_div(uint64_t num, uint64_t den, uint64_t* out);
int gfo_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint64_t* out);
int gfo_checked_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint32_t* out);
int gfo_plan_dense(const uint32_t* totals, uint64_t bins, uint32_t capacity, uint32_t* bin_base,
                   uint32_t* fills, uint64_t fills_cap, uint32_t* num_out);

/* ---- tile flattening (graph/TileDescriptor.hpp:25-30, flow/Execution.hpp:113-124,2377-2389) ---- */
typedef struct {
    uint32_t chunk_index;
    uint32_t tile_offset;
    uint32_t count;
} gfo_tile;
int gfo_tile_count(uint32_t fill, uint32_t tile_size, uint32_t* out);
int64_t gfo_flatten_tiles(const uint32_t* chunk_index, const uint32_t* fills, uint32_t n_chunks,
                          uint32_t tile_size, gfo_tile* out, uint64_t cap);

/* ---- classifiers on the path (examples/particle_feedback/KernelAxes.hpp:29-42 and the key
 *      classifiers of the kernel-level sweeps) ---- */
enum {
    GFO_CLS_KEY_MOD = 0,      /* bin = key % B                                     */
    GFO_CLS_ID_BALANCED = 1,  /* bin = id % B                        KernelAxes:29 */
    GFO_CLS_ID_ONEHOT = 2,    /* bin = 0                             KernelAxes:34 */
    GFO_CLS_ID_SKEWED = 3,    /* bin = id % 8 == 0 ? id % B : 0      KernelAxes:38 */
    GFO_CLS_KEY_UNMIX = 4     /* bin = unmix64(key) ^ salt (hash path, u64 keys)   */
};
uint32_t gfo_classify(int cls, uint64_t key, uint32_t bins, uint64_t salt);

/* ---- classify -> plan -> scatter (graph/ClassifyKernel.hpp:33-93, ScatterKernel.hpp:174-289) ---- */
/* Stable partition of n u32 keys (tile order) into B ports. counts[B] receives the per-port
 * totals, order[n] the input indices in port-major, input-stable order. Returns GFO_INVALID if a
 * classifier result is out of range (the counts[B] status slot of the reference). */
int gfo_partition_stable_u32(const uint32_t* keys, uint64_t n, uint32_t bins, int cls,
                             uint32_t* counts, uint32_t* order, int threads);
/* Same for u64 keys (hash path). */
int gfo_partition_stable_u64(const uint64_t* keys, uint64_t n, uint32_t bins, int cls, uint64_t salt,
                             uint32_t* counts, uint32_t* order, int threads);

/* Reference-structured CPU path over a chunk pool: classify every tile into bin_ids and counts,
 * plan, take output chunks from `free_chunks` in bin order, scatter with the per-tile range
 * reservation, and write the output descriptors. Used as the timed CPU baseline.
 * pool_in / pool_out: u32 columns of num_chunks * capacity slots. */
typedef struct {
    uint32_t chunk_index;
    uint32_t fill;
    uint32_t bin;
} gfo_out_desc;
int gfo_partition_pool_u32(const uint32_t* pool_in, uint32_t* pool_out, uint32_t capacity,
                           const gfo_tile* tiles, uint64_t n_tiles, uint32_t bins, int cls,
                           uint32_t* bin_ids, uint32_t* counts, const uint32_t* free_chunks,
                           uint64_t n_free, uint32_t* table, gfo_out_desc* outs, uint32_t* n_outs,
                           int threads);

/* ---- synthetic key distributions of the kernel-level sweeps ---- */
enum { GFO_DIST_UNIFORM = 0, GFO_DIST_ZIPF = 1, GFO_DIST_ONE_PORT = 2, GFO_DIST_ROUND_ROBIN = 3 };
uint32_t gfo_dist_purpose(int dist);
/* cdf[k] = sum_{r<=k} (r+1)^-s / sum_all, cdf[K-1] = 1 */
void gfo_zipf_cdf(double s, uint32_t k, double* cdf);
uint32_t gfo_zipf_sample(const double* cdf, uint32_t k, uint32_t draw);
void gfo_generate_keys_u32(int dist, uint64_t seed, uint64_t first_id, uint64_t n, uint32_t bins,
                           const double* cdf, uint32_t* keys, int threads);
/* hash-path records: key = mix64(r ^ salt), r ~ Zipf(cdf over K), weight = U(0,1] f32, tag = id */
void gfo_generate_records16(uint64_t seed, uint64_t first_id, uint64_t n, const double* cdf, uint32_t k,
                            uint64_t salt, uint64_t* keys, float* weights, uint32_t* tags, int threads);

/* ---- particle_feedback scalar model (tests/reference/ScalarModel.hpp:84-133) ---- */
int gfo_particle_scalar(uint64_t seed, uint64_t n, uint32_t max_visits, uint32_t* weights,
                        uint8_t* capped, uint64_t* capped_count, int threads);
/* sorted, run-length encoded histogram (examples/particle_feedback/ParticleTypes.hpp:206-219) */
uint64_t gfo_histogram_u32(uint32_t* values, uint64_t n, uint32_t* row_weight, uint64_t* row_count);

/* ---- photon_scattering analog scalar transport (tests/reference/ScalarTransport.hpp:87-209) ---- */
typedef struct {
    uint32_t event;
    uint32_t scatter_count;
    double x, y, z, ux, uy, uz;
} gfo_photon_terminal;
int gfo_photon_analog(uint64_t seed, uint64_t n, double thickness, double sigma_s, double sigma_a,
                      int isotropic, uint32_t max_scatters, gfo_photon_terminal* out, int threads);
/* The same transport with the bounded path trace (examples/photon_scattering/PhotonFunctors.hpp
 * :201-234 TraceWriter; records at :255 source, :364-369 scatter, :401-406 terminal as event + 1):
 * ids < min(n, trace_photons) keep up to trace_vertices vertices (vertices[id * trace_vertices + j]),
 * counts[id] the vertices kept, truncated[id] = 1 when one did not fit. */
typedef struct {
    uint32_t kind; /* 0 source, 1 scatter, 2 transmitted, 3 reflected, 4 absorbed, 5 capped */
    uint32_t scatter_count;
    double x, y, z, ux, uy, uz;
} gfo_trace_vertex;
int gfo_photon_analog_traced(uint64_t seed, uint64_t n, double thickness, double sigma_s, double sigma_a,
                             int isotropic, uint32_t max_scatters, gfo_photon_terminal* out, uint32_t trace_photons,
                             uint32_t trace_vertices, gfo_trace_vertex* vertices, uint32_t* counts,
                             uint32_t* truncated, int threads);

/* ---- weighted slab model of the FP32 Monte Carlo sweep (Henyey-Greenstein, implicit capture,
 *      Russian roulette); FP64 restatement, structure of ScalarTransport.hpp ---- */
typedef struct {
    double thickness, mu_a, mu_s, g, roulette_threshold, roulette_survival;
    uint32_t max_scatters, hist_bins;
} gfo_hg_params;
typedef struct {
    uint32_t event;         /* 1 transmitted, 2 reflected, 3 absorbed (roulette), 4 capped */
    uint32_t scatter_count;
    double weight;
    double cos_exit;        /* |uz| at exit */
} gfo_hg_terminal;
int gfo_photon_hg(uint64_t seed, uint64_t first_id, uint64_t n, const gfo_hg_params* p,
                  gfo_hg_terminal* out, double* refl_hist, double* trans_hist, uint64_t* event_counts,
                  int threads);

#ifdef __cplusplus
}
#endif
#endif
