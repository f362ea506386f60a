/* graphflow_b200: C ABI of the B200-native transform-batch hot path of graphFlow.
 *
 * Plain pointers and sizes only. Device pointers are marked `d_`, host pointers `h_`.
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 * Every kernel entry point is stream-ordered and asynchronous: it validates its arguments on
 * the host, enqueues its work and returns. Device-side failures (an invalid classifier result, a
 * checked updater overflow, an exhausted reservation, a wait that ran out of polls) are written
 * to the caller's device status word, which the caller zeroes before the batch and reads after
 * it, exactly like the reference's `Status` word and `counts[B]` status slot
 * (flow/Status.hpp:21-96, flow/Execution.hpp:2527-2547). No entry point throws.
 *
 * Reference paths below are inside the graphFlow project (include/graphFlow/...).
 */
#ifndef GRAPHFLOW_B200_H
#define GRAPHFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
/* 0..2 are the device StatusCode values of flow/Status.hpp:21-26; the rest are host-side. */
typedef enum gf_status {
    GF_OK = 0,
    GF_INVALID = 1,        /* StatusCode::invalid: bin >= B, bad payload                   */
    GF_OVERFLOW = 2,       /* StatusCode::overflow: checked updater or capacity overflow   */
    GF_ERR_ARGUMENT = 3,   /* std::invalid_argument of the reference (config/argument)     */
    GF_ERR_RANGE = 4,      /* std::overflow_error of the reference (32-bit limits)         */
    GF_ERR_LOGIC = 5,      /* std::logic_error of the reference (plan exceeds the bound)   */
    GF_ERR_CUDA = 6,       /* a CUDA runtime call failed                                   */
    GF_ERR_TIMEOUT = 7,    /* a bounded device wait gave up                                */
    GF_ERR_TABLE_FULL = 8  /* hash table of a tile is full (HashClassifyKernel.hpp:35-41)  */
} gf_status;

/* ---- data layouts ------------------------------------------------------------------------ */
/* One <= T slice of one pool chunk: graph/TileDescriptor.hpp:25-30. */
typedef struct gf_tile {
    uint32_t chunk_index;
    uint32_t tile_offset;
    uint32_t count;
} gf_tile;

/* One published output chunk: core/Chunk.hpp:33-37 (handle index, fill, bin). */
typedef struct gf_out_desc {
    uint32_t chunk_index;
    uint32_t fill;
    uint32_t bin;
} gf_out_desc;

/* Built-in classifiers. User functors cannot cross a C ABI; the C++ front end instantiates the
 * kernels with them directly. These ids cover the kernel-level sweeps and the kernel-axis
 * example classifiers (examples/particle_feedback/KernelAxes.hpp:29-42). */
enum {
    GF_CLS_KEY_MOD = 0,     /* bin = key % B                                  */
    GF_CLS_ID_BALANCED = 1, /* bin = id % B                                   */
    GF_CLS_ID_ONEHOT = 2,   /* bin = 0                                        */
    GF_CLS_ID_SKEWED = 3,   /* bin = id % 8 == 0 ? id % B : 0                 */
    GF_CLS_KEY_UNMIX = 4    /* bin = unmix64(key) ^ salt (u64 keys, hash path) */
};

/* Scatter strategies: core/ScatterMode.hpp (SharedStaging, Direct). */
enum { GF_SCATTER_SHARED = 0, GF_SCATTER_DIRECT = 1 };

/* Key distributions of the kernel-level sweeps. */
enum { GF_DIST_UNIFORM = 0, GF_DIST_ZIPF = 1, GF_DIST_ONE_PORT = 2, GF_DIST_ROUND_ROBIN = 3 };

/* ---- host-side planning (no device work) -------------------------------------------------- */

/* core/Reservation.hpp:35-50 outputChunkBound: R = min(n, ceil(n/C) + min(B, n) - 1). */
gf_status gf_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint64_t* h_out);

/* core/Reservation.hpp:61-71 checkedOutputChunkBound (narrowed to 32 bits). */
gf_status gf_checked_output_chunk_bound(uint64_t n, uint64_t capacity, uint64_t max_bins, uint32_t* h_out);

/* graph/DenseBinTable.hpp:39-77 planDenseBins. h_bin_base[bins], h_fills[fills_cap]. */
gf_status gf_plan_dense(const uint32_t* h_totals, uint32_t bins, uint32_t capacity, uint32_t* h_bin_base,
                        uint32_t* h_fills, uint32_t fills_cap, uint32_t* h_num_out);

/* graph/DenseBinTable.hpp:80-91 buildDenseTable: h_table[bins + num_out]. */
gf_status gf_build_dense_table(const uint32_t* h_bin_base, uint32_t bins, const uint32_t* h_chunk_indices,
                               uint32_t num_out, uint32_t* h_table);

/* flow/Execution.hpp:113-124 tileCount. */
gf_status gf_tile_count(uint32_t fill, uint32_t tile_size, uint32_t* h_out);

/* flow/Execution.hpp:2377-2389 flatten loop: one descriptor per <= tile_size slice of every
 * chunk, in chunk order. Returns GF_ERR_RANGE when `cap` descriptors do not suffice. */
gf_status gf_flatten_tiles(const uint32_t* h_chunk_index, const uint32_t* h_fills, uint32_t n_chunks,
                           uint32_t tile_size, gf_tile* h_tiles, uint32_t cap, uint32_t* h_n_tiles);

/* Tile sizes (particles per tile) the partition kernels of this build are compiled for. */
uint32_t gf_supported_tile_sizes(uint32_t* h_sizes, uint32_t cap);

/* Process-wide tuning knobs (no reference counterpart; used by the autotuner and the benchmark):
 *   "fused_coop" 1 (default) = gf_partition_fused_u32 uses the cooperative count/plan/scatter
 *                kernel where it applies (bins <= 64, tiles of at most 4096 particles,
 *                capacity % 4 == 0 and >= 4096, fewer than 2^32 pool slots, 16-byte aligned
 *                key columns); 0 = always the
 *                per-tile look-back kernel. Per-port counts, the plan and every port's sequence are
 *                identical either way; the cooperative kernel also takes the output chunks in plan
 *                order (table[B + f] = reserved[f]).
 *   "fused_coop_bulk" 1 (default) = for up to 16 ports the cooperative kernel writes each tile's
 *                port runs with bulk copies (shared -> global) when the scratch also holds one
 *                histogram per tile (gf_fused_scratch_bytes sizes it so); 0 = warp stores.
 *                Results are identical.
 *   "device_resident" 0 (default) = the flow entry points run their Flow with the host runner;
 *                1 = device-resident (Tuning::deviceResident): in waves, every node takes its whole
 *                input as one batch on one stream, output chunks come from a device-resident pool
 *                and each output chunk is appended on the device to the list of the node its port
 *                feeds; the host reads one block of list counters per wave. P, Q and the runner
 *                options do not apply; partitions run the fused dense kernel (the kernel workload's
 *                plain, direct-scatter and hash-path forms keep the host runner). Results are
 *                identical.
 *   "device_coop" 1 (default) = in device-resident runs and gf_run_dense_chain_device, a partition
 *                batch of at least 64 tiles and up to 64 ports runs the cooperative count -> grid
 *                barrier -> scatter kernel (bins kept from the count pass); 0 = the per-tile
 *                look-back kernel. Results are identical.
 *   "runner_batched" 1 (default) = the flow entry points (gf_run_particle_feedback,
 *                gf_run_dense_chain, gf_run_photon) let a sink take up to "sink_batch_chunks"
 *                ready chunks per launch and dispatch every idle node in one scheduler iteration;
 *                0 = the reference runner's one-chunk sinks and one dispatch per iteration.
 *                Results are identical.
 *   "sink_batch_chunks" 1..256 (default 256) = chunks per sink launch in the batched runner.
 *   "group_partitions" 1 (default) = with "runner_batched", the flow entry points
 *                (gf_run_dense_chain, gf_run_particle_feedback, gf_run_kernel_axes, gf_run_photon)
 *                run their fused partition nodes of one type as one partition group (a group may be
 *                one node): one launch drains every member node's ready batches, each of at most Q
 *                chunks (sched/GraphRunner.hpp:985-1133 launches once per node batch); 0 = one
 *                runner node per partition node. Results are identical.
 *   "hash_persistent" 1 (default) = gf_classify_hash_r16 and gf_scatter_hash_r16 use the
 *                persistent kernels (one shared-memory counter per port and CTA for the count;
 *                the scatter groups each tile's records of ports below 2048 by port and places
 *                rarer ports one record at a time); 0 = the per-tile open-addressing table
 *                kernels (graph/BinTable.hpp design). Counts, the plan and every port's record
 *                multiset are identical; the order inside a port is arrival order either way.
 *   "spin_limit" polls (default 2^20; 0 or less restores it) = how often a wait between CTAs of the
 *                fused partition kernels polls before it gives up with GF_ERR_TIMEOUT (a short
 *                limit lets a test make a wait run out); sets a device variable, so it needs a GPU.
 * Unknown names and out-of-range values return GF_ERR_ARGUMENT. */
gf_status gf_set_tuning(const char* name, int value);

/* ---- dense partition: the reference's two-launch form --------------------------------------- */

/* flow/Execution.hpp:870-954 PartitionClassifyKernel (graph/ClassifyKernel.hpp:33-93) over a u32
 * key column in the fixed pool layout (slot = chunk_index * capacity + offset).
 * Writes d_bin_ids[slot] and accumulates d_counts[0..bins) (caller zeroes them);
 * d_counts[bins] is the status slot (set to 1 on an invalid bin). */
gf_status gf_classify_dense_u32(void* stream, const uint32_t* d_keys, uint32_t capacity, uint64_t pool_slots,
                                const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size, uint32_t bins,
                                int classifier, uint32_t* d_bin_ids, uint32_t* d_counts, uint32_t* d_status);

/* flow/Execution.hpp:985-1189 PartitionScatterKernel (graph/ScatterKernel.hpp:174-289).
 * d_table = [binBase[bins], chunkIndex[R]] (buildDenseTable layout); d_next[bins] zeroed by the
 * caller; after the launch d_next[b] == totals[b] (finalise, Execution.hpp:2715-2725).
 * d_keys_in and d_keys_out may be the same pool column (inputs and outputs are distinct chunks). */
gf_status gf_scatter_dense_u32(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out, uint32_t capacity,
                               uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size,
                               uint32_t bins, const uint32_t* d_bin_ids, const uint32_t* d_table, uint32_t* d_next,
                               uint32_t* d_counts, int mode, uint32_t* d_status);

/* ---- dense partition: single-pass fused classify -> scan -> scatter -------------------------- */

/* Scratch bytes gf_partition_fused_u32 needs for n_tiles tiles and `bins` ports. */
gf_status gf_fused_scratch_bytes(uint32_t n_tiles, uint32_t bins, uint64_t* h_bytes);

/* One launch replaces classify + host plan + scatter (flow/Execution.hpp:2363-2642): per tile,
 * classify, rank stably inside the tile, obtain each port's exclusive prefix across tiles with a
 * decoupled look-back, take output chunks on first touch from the caller's reservation
 * d_reserved[n_reserved] (the outputChunkBound credit of GraphRunner.hpp:1014-1037), and write
 * the payload. Positions inside a port follow the input order (stable partition).
 * Outputs: d_totals[bins] and d_port_chunks[bins * max_chunks_per_port] (epoch-tagged chunk
 * index of port b's k-th chunk; gf_fused_finish turns them into the reference's table).
 * d_scratch (gf_fused_scratch_bytes, 16-byte aligned) must be zero-filled before its first use
 * and then stays owned by this call site: it carries the launch epoch from one launch to the
 * next, which lets the launch be replayed from a CUDA graph. Launches sharing one scratch must
 * not overlap on the GPU. */
gf_status gf_partition_fused_u32(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out, uint32_t capacity,
                                 uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size,
                                 uint32_t bins, int classifier, const uint32_t* d_reserved, uint32_t n_reserved,
                                 uint32_t* d_totals, unsigned long long* d_port_chunks, uint32_t max_chunks_per_port,
                                 void* d_scratch, uint64_t scratch_bytes, uint32_t* d_status);

/* Builds the reference-layout results of the last fused launch on `d_scratch` on the device:
 * d_table[bins + R] ([binBase, chunkIndex], DenseBinTable.hpp:80-91), d_descs[R] output
 * descriptors in bin order with their fills (Execution.hpp:2558-2581), and d_num_out[1] = R. */
gf_status gf_fused_finish(void* stream, const uint32_t* d_totals, const unsigned long long* d_port_chunks,
                          uint32_t bins, uint32_t capacity, uint32_t max_chunks_per_port, const void* d_scratch,
                          uint32_t* d_table, gf_out_desc* d_descs, uint32_t desc_cap, uint32_t* d_num_out,
                          uint32_t* d_status);

/* gf_partition_fused_u32 followed by gf_fused_finish, in one launch (no reference counterpart;
 * the pair above restates flow/Execution.hpp:2363-2642 + 2558-2590): the cooperative kernel writes
 * d_table, d_descs and d_num_out during its plan, the per-tile kernel in its last CTA. Arguments,
 * outputs and scratch rules are those of the two calls; results are identical to them. */
gf_status gf_partition_fused_full_u32(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out,
                                      uint32_t capacity, uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles,
                                      uint32_t tile_size, uint32_t bins, int classifier, const uint32_t* d_reserved,
                                      uint32_t n_reserved, uint32_t* d_totals, unsigned long long* d_port_chunks,
                                      uint32_t max_chunks_per_port, void* d_scratch, uint64_t scratch_bytes,
                                      uint32_t* d_table, gf_out_desc* d_descs, uint32_t desc_cap,
                                      uint32_t* d_num_out, uint32_t* d_status);

/* No counterpart in the reference. The fused partition plus its device finish for callers that
 * cannot allocate device memory at this point: a host runtime that gives all device memory to
 * its own pool at start-up and forbids cudaMalloc afterwards, or a latency-critical path that
 * cannot afford the device synchronisation cudaMalloc/cudaFree may cause. Arguments and outputs
 * are those of gf_partition_fused_u32 followed by gf_fused_finish; the caller still provides
 * every input and output buffer. The scratch is a fixed 8 MiB array inside the library, held by
 * every GPU that loads it until the process exits, so one batch may use at most
 * 64 + 8 x tiles x ports <= 8 MiB (e.g. 24,415 tiles of 4096 keys x 32 ports); larger batches
 * get GF_ERR_RANGE and a message from gf_last_error(). Devices 0..63 are served (others get
 * GF_ERR_RANGE and a message). The first call on a device sets the array up (takes its device
 * address, zeroes its 64-byte control block with a synchronous memset); make that first call
 * before any stream capture. The set-up holds for the life of the process's primary context on
 * that device: after cudaDeviceReset (or anything else that destroys the primary context) this
 * entry point must not be called again in the process. Every call on a device shares the array
 * and it keeps the last call's contents: calls that overlap on the GPU race, so order them on
 * one stream or synchronise between them. The finish outputs (d_table, d_num_out, d_descs) are
 * checked before anything runs. No call allocates or frees device memory. */
gf_status gf_partition_fused_u32_noalloc(void* stream, const uint32_t* d_keys_in, uint32_t* d_keys_out,
                                         uint32_t capacity, uint64_t pool_slots, const gf_tile* d_tiles,
                                         uint32_t n_tiles, uint32_t tile_size, uint32_t bins, int classifier,
                                         const uint32_t* d_reserved, uint32_t n_reserved, uint32_t* d_totals,
                                         unsigned long long* d_port_chunks, uint32_t max_chunks_per_port,
                                         uint32_t* d_table, gf_out_desc* d_descs, uint32_t desc_cap,
                                         uint32_t* d_num_out, uint32_t* d_status);

/* ---- generic partition and transform over registered record types ---------------------------
 * The entry points the reference's stages bind for any payload (flow/Execution.hpp:709-776
 * TransformKernel, :870-954 classify, :985-1189 scatter), over a column descriptor instead of the
 * u32 key column. User functors cannot cross a C ABI: each record type below and each classifier,
 * updater and transform id is a compile-time instantiation of the same kernels the C++ Flow runs
 * (the explicit instantiation table of gf_generic.cu). A record/functor pair the table does not
 * list returns GF_ERR_ARGUMENT. */
enum {
    GF_REC_U32 = 0,      /* {u32 key}                                                          */
    GF_REC_KEYREC = 1,   /* {u32 id, u32 key} (the dense chain's record)                       */
    GF_REC_PARTICLE = 2, /* {u64 id, u32 property, u32 weight, u32 visit}: particle_feedback's
                          * record (examples/particle_feedback/ParticleTypes.hpp:35-47); AoS
                          * slots are 24 bytes (the C struct's alignment padding)             */
    GF_REC_R16 = 3       /* {u64 key, f32 weight, u32 tag} (the hash path's record)            */
};
/* Device columns of a pool of one record type: SoA = column[i] holds field i (in the record's
 * field order above) of every slot; AoS = column[0] holds the slots. */
typedef struct gf_columns {
    int32_t record; /* GF_REC_* */
    int32_t layout; /* GF_LAYOUT_SOA / GF_LAYOUT_AOS */
    void* column[4];
} gf_columns;

/* Further registered classifiers (GF_CLS_KEY_MOD and GF_CLS_ID_* above apply to the records with
 * a key / an id field): */
enum {
    GF_CLS_FEEDBACK_FILTER = 16, /* particle_feedback Filter: bin = draw >= property ? 1 : 0
                                  * (ParticleFunctors.hpp FilterByProperty)                       */
    GF_CLS_FEEDBACK_SELECT = 17  /* A/B: draw < 2^31 ? sink (0) : visit < max_visits ? feedback (1)
                                  * : capped (2) (SelectOutcome)                                  */
};
/* Registered updaters, applied to every payload the scatter emits (purpose + 1 engine). */
enum {
    GF_UPD_NONE = 0,
    GF_UPD_SET_BIN = 1,  /* weight = bin (KernelAxes.hpp:80-106, particle records)               */
    GF_UPD_FEEDBACK = 2  /* on bin 1 (feedback): checked weight += increment, visit += 1
                          * (ParticleFunctors.hpp UpdateWeight; overflow sets GF_OVERFLOW)        */
};
/* Registered transforms (out-of-place, dense concatenation of the batch). */
enum {
    GF_XF_IDENTITY = 0,   /* copy                                                              */
    GF_XF_ADD_WEIGHT = 1  /* particle records: checked weight += increment, visit += 1            */
};
/* Functor parameters: seed (the keyed RNG streams, rng/ParticleRng.hpp), the node's stream
 * purpose (functor purpose; its updater uses purpose + 1), and the functor's constants. */
typedef struct gf_functor_params {
    uint64_t seed;
    uint32_t purpose;
    uint32_t max_visits; /* GF_CLS_FEEDBACK_SELECT */
    uint32_t increment;  /* GF_UPD_FEEDBACK, GF_XF_ADD_WEIGHT */
    uint32_t pad;
} gf_functor_params;

/* One <= tile slice of one input chunk and its position in the batch's dense output (the
 * reference's transform tile: TileDescriptor plus outPosition, Execution.hpp:709-776). */
typedef struct gf_move_tile {
    uint32_t in_chunk;
    uint32_t in_offset;
    uint32_t count;
    uint32_t out_pos;
} gf_move_tile;

/* flow/Execution.hpp:870-954 PartitionClassifyKernel for any registered record: per-port counts
 * in d_counts[0..bins) and the status slot d_counts[bins] (a result >= bins), d_bin_ids per slot. */
gf_status gf_classify_dense(void* stream, const gf_columns* h_cols, uint32_t capacity, uint64_t pool_slots,
                            const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size, uint32_t bins,
                            int classifier, const gf_functor_params* h_params, uint32_t* d_bin_ids,
                            uint32_t* d_counts, uint32_t* d_status);

/* flow/Execution.hpp:985-1189 PartitionScatterKernel for any registered record: every field of
 * each payload moves from h_in's slot to the planned slot of h_out (table = [binBase, chunkIndex]
 * of the plan, next[bins] zeroed), the updater applied on the way. mode GF_SCATTER_SHARED or
 * _DIRECT. h_in and h_out may describe the same columns. */
gf_status gf_scatter(void* stream, const gf_columns* h_in, const gf_columns* h_out, uint32_t capacity,
                     uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size, uint32_t bins,
                     const uint32_t* d_bin_ids, const uint32_t* d_table, uint32_t* d_next, uint32_t* d_counts,
                     int mode, int updater, const gf_functor_params* h_params, uint32_t* d_status);

/* flow/Execution.hpp:709-776 TransformKernel: input item i of tile t goes, transformed, to dense
 * output position t.out_pos + i, i.e. chunk d_out_chunks[pos / C] at offset pos % C. */
gf_status gf_transform(void* stream, const gf_columns* h_in, const gf_columns* h_out, uint32_t capacity,
                       uint64_t pool_slots, const gf_move_tile* d_tiles, uint32_t n_tiles,
                       const uint32_t* d_out_chunks, uint32_t n_out, int transform,
                       const gf_functor_params* h_params, uint32_t* d_status);

/* gf_partition_fused_full_u32 for any registered record, classifier and updater: one fused
 * classify -> plan -> scatter launch plus its device finish (the per-tile look-back kernel;
 * ports < 4096), output chunks from the caller's reservation, per-port sequences in input order.
 * Scratch: gf_fused_scratch_bytes(n_tiles, bins). */
gf_status gf_partition_fused(void* stream, const gf_columns* h_cols, uint32_t capacity, uint64_t pool_slots,
                             const gf_tile* d_tiles, uint32_t n_tiles, uint32_t bins, int classifier, int updater,
                             const gf_functor_params* h_params, const uint32_t* d_reserved, uint32_t n_reserved,
                             uint32_t* d_totals, unsigned long long* d_port_chunks, uint32_t max_chunks_per_port,
                             void* d_scratch, uint64_t scratch_bytes, uint32_t* d_table, gf_out_desc* d_descs,
                             uint32_t desc_cap, uint32_t* d_num_out, uint32_t* d_status);

/* ---- hash partition of 16-byte records (large port counts) ---------------------------------- */

/* Columns of the 16-byte record {u64 key, f32 weight, u32 tag}: SoA uses key/weight/tag, AoS
 * uses `records` (16-byte aligned, 16 bytes per slot). Pointers are device pointers; the struct
 * itself is passed from host memory. */
typedef struct gf_rec16_columns {
    uint64_t* key;
    float* weight;
    uint32_t* tag;
    void* records;
} gf_rec16_columns;
enum { GF_LAYOUT_SOA = 0, GF_LAYOUT_AOS = 1 };
/* gf_run_particle_feedback only: the graph over a graphFlow::Record payload (named attributes, one
 * device column each; examples/particle_feedback/ParticleTypes.hpp:20-47 in the reference). */
enum { GF_LAYOUT_RECORD = 2 };

/* Tile sizes the hash kernels are compiled for (the shared table has 2 x tile entries). */
uint32_t gf_supported_hash_tile_sizes(uint32_t* h_sizes, uint32_t cap);

/* flow/Execution.hpp:1208-1307 PartitionHashClassifyKernel (graph/HashClassifyKernel.hpp:35-117).
 * bin = unmix64(key) ^ salt (< bins, else the status slot d_counts[bins] is set). A shared-memory
 * open-addressing table aggregates the tile (graph/BinTable.hpp:29-137). d_bin_ids may be NULL
 * (nothing stored: the scatter then recomputes the bin from the key). */
gf_status gf_classify_hash_r16(void* stream, const gf_rec16_columns* h_cols, int layout, uint32_t capacity,
                               uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles, uint32_t tile_size,
                               uint32_t bins, uint64_t salt, uint32_t* d_bin_ids, uint32_t* d_counts,
                               uint32_t* d_status);

/* flow/Execution.hpp:1336-1502 PartitionHashScatterKernel (graph/HashScatterKernel.hpp:34-183):
 * rebuild the tile table from d_bin_ids (or recompute bins when NULL), reserve one range per
 * occupied entry on d_next[bin], write through d_table = [binBase[bins], chunkIndex[R]]. */
gf_status gf_scatter_hash_r16(void* stream, const gf_rec16_columns* h_in, const gf_rec16_columns* h_out, int layout,
                              uint32_t capacity, uint64_t pool_slots, const gf_tile* d_tiles, uint32_t n_tiles,
                              uint32_t tile_size, uint32_t bins, uint64_t salt, const uint32_t* d_bin_ids,
                              const uint32_t* d_table, uint32_t* d_next, uint32_t* d_counts, uint32_t* d_status);

/* Device form of the exact plan (graph/DenseBinTable.hpp:39-91 + the acquisition loop of
 * flow/Execution.hpp:2558-2590) so that classify -> plan -> scatter needs no host round trip:
 * from d_counts[bins + 1] (classify output; a set status slot aborts the plan) and a
 * reservation d_reserved[n_reserved], writes d_table[bins + R], d_descs[R] (bin order, chunk
 * (b, k) = d_reserved[binBase[b] + k]), d_num_out[1] = R, and zeroes d_next[bins]. */
gf_status gf_plan_device(void* stream, const uint32_t* d_counts, uint32_t bins, uint32_t capacity,
                         const uint32_t* d_reserved, uint32_t n_reserved, uint32_t* d_table, gf_out_desc* d_descs,
                         uint32_t desc_cap, uint32_t* d_num_out, uint32_t* d_next, uint32_t* d_status);

/* ---- synthetic sources ---------------------------------------------------------------------- */

/* Zipf(s) cumulative table over k ranks on the host: cdf[r] = sum_{i<=r} (i+1)^-s / total. */
gf_status gf_zipf_cdf(double s, uint32_t k, double* h_cdf);

/* Fills d_keys[0..n) with the key distribution `dist` at stream positions
 * (first_id + i, 0, 0x100 + dist): uniform = first Philox draw, zipf = inverse CDF of that draw
 * over d_cdf[bins], one_port = 0, round_robin = first_id + i. */
gf_status gf_generate_keys_u32(void* stream, int dist, uint64_t seed, uint64_t first_id, uint64_t n, uint32_t bins,
                               const double* d_cdf, uint32_t* d_keys);

/* Fills slots [0, n) of the record columns: rank r ~ Zipf over d_cdf[k], key = mix64(r ^ salt),
 * weight = U(0,1] (f32), tag = first_id + i; stream position (first_id + i, 0, 0x110). */
gf_status gf_generate_records16(void* stream, uint64_t seed, uint64_t first_id, uint64_t n, const double* d_cdf,
                                uint32_t k, uint64_t salt, const gf_rec16_columns* h_cols, int layout);

/* ---- device policy: default C, P and T (core/DevicePolicy.hpp:344-614 makeDevicePolicy) ------- */

/* The fields of a device the policy reads (alpaka DeviceProperties subset). */
typedef struct gf_device_props {
    uint32_t sms;
    uint32_t warp_size;
    uint32_t max_threads_per_block;
    uint32_t max_blocks_per_grid;
    uint32_t shared_mem_per_block; /* bytes, default per-block limit */
    uint64_t global_mem_bytes;
} gf_device_props;

typedef struct gf_policy {
    uint32_t chunk_capacity; /* C */
    uint32_t live_particles; /* P */
    uint32_t tile_size;      /* T */
    uint32_t live_explicit;  /* P came from the caller */
    uint64_t budget_bytes;   /* payload budget the clamps used */
} gf_policy;

/* C, P and T for a run of n particles on h_props (NULL: the current CUDA device), with the
 * reference's rules: T = 128 rounded to the warp and capped by a 2T-entry hash table in shared
 * memory; C = waves x SMs x 4 x T capped by 8192 (or the explicit C), the grid, n and the payload
 * budget, rounded to T; P = min(n, ratio x C) clamped so P x C x slot_bytes fits the budget, the
 * budget being min(global memory / 8, 3 GiB) unless budget_bytes is given. 0 in chunk_capacity,
 * live_particles, tile_size or budget_bytes means "derive"; live_per_chunk 0 means the
 * reference's direct-call ratio 2 (the Flow uses 8); slot_bytes 0 means 24. An impossible request
 * (explicit P above n or beyond the budget, explicit C above the maximum or the grid) returns
 * GF_ERR_ARGUMENT with the reason in gf_last_error(). */
gf_status gf_device_policy(const gf_device_props* h_props, uint64_t n, uint32_t chunk_capacity,
                           uint32_t live_particles, uint32_t tile_size, uint32_t live_per_chunk,
                           uint64_t budget_bytes, uint64_t slot_bytes, gf_policy* h_out);

/* ---- whole flows through the C++ front end (Flow / GraphRunner) ------------------------------ */
/* The flow entry points (gf_run_particle_feedback*, gf_run_dense_chain, gf_run_photon) and the
 * request server run on the calling thread's current CUDA device (cudaSetDevice). A chunk_capacity
 * or live_particles of 0 takes the device policy's C or P (gf_device_policy on that device with the
 * Flow's ratio P/C = 8 and the flow's slot size). */

/* Counters of one run (sched/GraphRunner.hpp:154-252 SchedulerStats, subset). */
typedef struct gf_flow_stats {
    uint64_t completed_batches;
    uint64_t partition_batches;
    uint64_t kernel_launches;
    uint64_t loop_iterations;
    uint64_t generated;
    uint64_t sunk;
    uint32_t pool_chunks;
    uint32_t peak_live_chunks;
    uint32_t peak_reserved_chunks;
    uint32_t peak_ready_chunks;
    double seconds;       /* wall time of the entry point's run, Flow built and destroyed included */
    double setup_seconds; /* of it: the Flow's storage, stages and runner built */
    double loop_seconds;  /* of it: the scheduler loop (the rest: final synchronisation, teardown) */
    uint64_t partition_launches; /* launches that ran partition batches; a partition group runs many
                                  * nodes' batches per launch (partition_batches counts the batches) */
} gf_flow_stats;

/* examples/particle_feedback/KernelAxes.hpp:115-214 runKernelAxes: Generate -> one partition with
 * `bins` ports (64, 1024, 4096 or 65536; the classifier is distributionBin of the particle id) ->
 * one sink on every port, the updater writing the port into the weight: h_weights[n] = each
 * particle's port. distribution GF_KDIST_*; scatter_mode GF_SCATTER_SHARED / _DIRECT (direct only
 * with fused = 0 and the dense path: one device atomic per particle in the plain form's scatter);
 * hash_path != 0 partitions through the per-tile hash tables (the bin path 65536 ports always take);
 * sparse needs bins >= 1024. Errors as gf_run_particle_feedback. */
enum { GF_KDIST_BALANCED = 0, GF_KDIST_ONEHOT = 1, GF_KDIST_SKEWED = 2, GF_KDIST_SPARSE = 3 };
gf_status gf_run_kernel_axes(uint64_t seed, uint64_t n, uint32_t bins, int distribution, int scatter_mode,
                             int hash_path, uint32_t chunk_capacity, uint32_t live_particles, uint32_t batch_chunks,
                             int fused, uint32_t* h_weights, gf_flow_stats* h_stats);

/* A transform restricted to an attribute subset (flow/Flow.hpp:235-242 transform<Set<Tags...>>):
 * Generate (the particle_feedback source over a Record payload) -> transform<Set<WeightTag,
 * VisitTag>> adding `increment` to the weight and 1 to the visit -> sink. h_weights[id] and
 * h_visits[id] receive every particle's weight (= increment) and visit (= 1). No reference entry
 * point; it runs the front end's attribute-subset transform. Errors as gf_run_particle_feedback. */
gf_status gf_run_set_transform(uint64_t seed, uint64_t n, uint32_t increment, uint32_t chunk_capacity,
                               uint32_t live_particles, uint32_t batch_chunks, uint32_t* h_weights,
                               uint32_t* h_visits, gf_flow_stats* h_stats);

/* The same feedback graph with the same functors and RNG streams, run as one per-particle kernel
 * (every particle carried from the source to its sink by one thread, no batches): h_weights and
 * h_capped as gf_run_particle_feedback, identical values. No reference counterpart as an entry
 * point; it is the fused execution of runParticleFeedback's graph. */
gf_status gf_run_particle_feedback_kernel(uint64_t seed, uint64_t n, uint32_t max_visits, uint32_t* h_weights,
                                          uint32_t* h_capped, gf_flow_stats* h_stats);

/* ---- device histogram ---------------------------------------------------------------------- */

/* examples/particle_feedback/ParticleTypes.hpp:206-219 histogramOf (sort + run-length encoding) on
 * the GPU: the sorted (value, count) rows of d_values[n], n <= 2^31. The sort is a radix sort whose
 * passes are the stable cooperative partition (6-bit digits; digits equal for every value are
 * skipped). d_row_values / d_row_counts need room for n rows; *d_num_rows receives the row count,
 * failures go to the caller-zeroed *d_status. The call waits once on `stream` (after one reduction
 * that selects the passes); everything else is enqueued. Scratch: gf_histogram_scratch_bytes,
 * 256-byte aligned. */
gf_status gf_histogram_scratch_bytes(uint64_t n, uint64_t* h_bytes);
gf_status gf_histogram_u32(void* stream, const uint32_t* d_values, uint64_t n, void* d_scratch,
                           uint64_t scratch_bytes, uint32_t* d_row_values, unsigned long long* d_row_counts,
                           uint32_t* d_num_rows, uint32_t* d_status);

/* ---- request server (continuous batching; no reference counterpart) -------------------------- */

/* Whole-flow request kinds: the particle_feedback graph (64 visits), the weighted FP32 photon slab
 * (L=1, mu_s=10, mu_a=0.1, g=0.9, roulette below 1e-4), and a two-node dense classify chain over
 * uniform u32 keys (bins in {2, 8, 32}, C=8192). */
enum { GF_REQ_PARTICLE_FEEDBACK = 0, GF_REQ_PHOTON = 1, GF_REQ_DENSE_CHAIN = 2 };
/* GF_SERVE_PLAIN: one request at a time in arrival order through the C++ Flow with plain partitions
 * and the reference runner. GF_SERVE_BATCHED: continuous batching, every admitted request's whole
 * flow on the device on its own stream, admitted while others run as stream slots and device
 * memory (an arena capped at memory_cap_bytes) free up. GF_SERVE_FLOW_DEVICE: one request at a
 * time through the same Flow graphs as GF_SERVE_PLAIN, run device-resident (knob
 * "device_resident"). */
enum { GF_SERVE_PLAIN = 0, GF_SERVE_BATCHED = 1, GF_SERVE_FLOW_DEVICE = 2 };

typedef struct gf_request {
    uint32_t kind;    /* GF_REQ_* */
    uint32_t bins;    /* dense chain: 2, 8 or 32; ignored otherwise */
    uint64_t n;       /* particles (photons) of the request, < 2^32 */
    uint64_t seed;
    double arrival_s; /* arrival, seconds after the stream starts; non-decreasing */
} gf_request;

typedef struct gf_request_result {
    double admit_s;  /* when the request was admitted (plain form: when it started) */
    double done_s;   /* when its result was on the host; latency = done_s - arrival_s */
    uint64_t digest; /* order-independent 64-bit digest of the per-particle result */
    uint32_t status; /* gf_status of the request (GF_ERR_RANGE: larger than the memory cap) */
    uint32_t pad;
} gf_request_result;

typedef struct gf_serve_stats {
    double seconds;         /* stream start to the last completion */
    uint64_t peak_bytes;    /* most device memory granted to requests at once */
    uint32_t peak_inflight; /* most requests on the device at once */
    uint32_t pad;
} gf_serve_stats;

/* Serves n_requests requests (sorted by arrival) and fills h_results[n_requests]. A request's
 * digest is the same in either mode and alone or in a mix. max_inflight: 1..256 streams.
 * Errors: GF_ERR_ARGUMENT before any work; per-request failures in h_results[i].status. */
gf_status gf_serve(const gf_request* h_requests, uint32_t n_requests, int mode, uint64_t memory_cap_bytes,
                   uint32_t max_inflight, gf_request_result* h_results, gf_serve_stats* h_stats);

/* The kernel-level dense sweep through the public Flow (flow/Flow.hpp:49-754 with the
 * reference's runner semantics, sched/GraphRunner.hpp): Generate -> `nodes` (1..4) chained
 * partition nodes -> sink. Records are {u32 id, u32 key}; keys are gf_generate_keys_u32's for the
 * same seed and distribution (zipf_s is the Zipf exponent); node i sends a key to port
 * (key >> 8 i) mod bins, bins in {2, 8, 32, 64}; every port of a node feeds the next node and the
 * last node feeds the sink. h_port_of[n] (optional) receives each particle's final port
 * (0xFFFFFFFF if it never reached the sink). chunk_capacity = C, live_particles = P (0: default),
 * batch_chunks = Q, fused != 0: one fused launch per partition batch, layout GF_LAYOUT_SOA/_AOS.
 * Errors as gf_run_particle_feedback. */
gf_status gf_run_dense_chain(uint64_t seed, uint64_t n, uint32_t bins, uint32_t nodes, int dist, double zipf_s,
                             uint32_t chunk_capacity, uint32_t live_particles, uint32_t batch_chunks, int fused,
                             int layout, uint32_t* h_port_of, gf_flow_stats* h_stats);

/* ---- device-resident chunk pool ----------------------------------------------------------------
 * The host pool's free list, per-chunk ledger and reservation credits (core/ChunkPool.hpp:88-190,
 * core/ChunkLedger.hpp:33-150, sched/GraphRunner.hpp:1014-1037) in device memory, for flows whose
 * nodes run on the device without host round trips. One allocation of gf_device_pool_bytes(S)
 * bytes (16-byte aligned) holds chunks 0..S-1; every operation is one kernel on `stream`, and the
 * operations on one pool must be stream-ordered.
 *   acquire  pops k chunks into d_ids[k] in the host pool's order (a fresh pool hands out 0, 1, ...;
 *            the chunk released last comes out first). Fewer than k free: GF_OVERFLOW in *d_status
 *            and in the pool, nothing taken, d_ids filled with 0xFFFFFFFF.
 *   settle   after a batch that reserved d_reserved[reserved_n] (its outputChunkBound, from one
 *            acquire) and used the first *d_used (or `used` when d_used is NULL) of them: the
 *            unused ones go back exactly where they were, then the input chunks
 *            d_in[j * in_stride], j < *d_in_count (or in_count), are released (in_stride 1 for an
 *            id array, 3 for the chunk_index field of gf_out_desc records). A chunk that is not
 *            live, out of range, named twice or one of the unused reservations, or unused
 *            reservations no longer at the front of the free list: GF_INVALID, nothing changed.
 * A chunk's ledger word is generation << 1 | live; releases step the generation. */
typedef struct gf_device_pool_stats {
    uint32_t num_chunks;
    uint32_t free_chunks;
    uint32_t peak_live; /* most chunks out of the pool at once */
    uint32_t status;    /* GF_OK or the first failed operation's code */
    uint64_t acquired;  /* chunks acquired over the pool's life (returned reservations excluded) */
    uint64_t released;
} gf_device_pool_stats;

gf_status gf_device_pool_bytes(uint32_t num_chunks, uint64_t* h_bytes);
gf_status gf_device_pool_init(void* stream, void* d_pool, uint32_t num_chunks);
gf_status gf_device_pool_acquire(void* stream, void* d_pool, uint32_t k, uint32_t* d_ids, uint32_t* d_status);
gf_status gf_device_pool_settle(void* stream, void* d_pool, const uint32_t* d_reserved, uint32_t reserved_n,
                                const uint32_t* d_used, uint32_t used, const uint32_t* d_in, uint32_t in_stride,
                                const uint32_t* d_in_count, uint32_t in_count, uint32_t* d_status);
/* Synchronises `stream` and reads the pool's counters. */
gf_status gf_device_pool_read(void* stream, const void* d_pool, gf_device_pool_stats* h_stats);

/* The same dense chain as gf_run_dense_chain (same records, keys, ports and results) run entirely on
 * the device: one stream, the host enqueues every launch up front and synchronises once. Each node
 * is one fused partition launch over its whole input, with its output chunks reserved from a
 * device-resident pool (outputChunkBound per node, the unused ones returned and the node's input
 * chunks released after it): C = 8192, tiles of 4096, pool S = max(ceil(n / C), bound) + bound
 * chunks. h_port_of[n], h_node_totals[nodes * bins] (node i's per-port counts), h_pool (the pool's
 * counters at the end: every chunk free again) and h_stats are optional; h_stats->loop_seconds is
 * the device time from the first launch to the last. Errors as gf_run_dense_chain. */
gf_status gf_run_dense_chain_device(uint64_t seed, uint64_t n, uint32_t bins, uint32_t nodes, int dist,
                                    double zipf_s, uint32_t* h_port_of, uint32_t* h_node_totals,
                                    gf_device_pool_stats* h_pool, gf_flow_stats* h_stats);

/* examples/particle_feedback/ParticleFeedback.hpp:41-108 runParticleFeedback: the
 * Generate -> Filter -> {A, B} -> sink feedback graph with the example's functors, on the GPU.
 * h_weights[n] receives each particle's final weight (0xDEADBEEF if it never reached a sink),
 * h_capped[n] is 1 for particles stopped by the visit cap. layout: GF_LAYOUT_SOA / _AOS, or
 * GF_LAYOUT_RECORD for the same graph written over a Record payload (identical results).
 * fused != 0 runs each partition batch as one fused launch, else classify + host plan + scatter.
 * Errors: GF_ERR_ARGUMENT (configuration), GF_ERR_RANGE (32/16-bit stream limits),
 * GF_INVALID / GF_OVERFLOW (a batch failed), GF_ERR_TIMEOUT (scheduler stall), GF_ERR_CUDA;
 * gf_last_error() describes the last failure of the calling thread. */
gf_status gf_run_particle_feedback(uint64_t seed, uint64_t n, uint32_t max_visits, uint32_t chunk_capacity,
                                   uint32_t live_particles, uint32_t batch_chunks, int fused, int layout,
                                   uint32_t* h_weights, uint32_t* h_capped, gf_flow_stats* h_stats);

/* photon_scattering (examples/photon_scattering/PhotonScattering.hpp:37-181 topology).
 * model GF_PHOTON_ANALOG: the reference example (absorption terminal, forward or isotropic
 * scattering). model GF_PHOTON_WEIGHTED: Henyey-Greenstein g, implicit capture, Russian roulette
 * below roulette_threshold (survival probability roulette_survival), exit-weight histograms over
 * hist_bins bins of |cos theta| for reflection and transmission. */
typedef struct gf_photon_params {
    double thickness, sigma_s, sigma_a, g, roulette_threshold, roulette_survival;
    uint32_t max_scatters;
    uint32_t hist_bins;
    int model;     /* GF_PHOTON_ANALOG or GF_PHOTON_WEIGHTED */
    int isotropic; /* analog model: isotropic (1) or forward (0) scattering */
    int fp64;      /* 1: double arithmetic, 0: float */
} gf_photon_params;
enum { GF_PHOTON_ANALOG = 0, GF_PHOTON_WEIGHTED = 1 };
enum { GF_EXEC_FLOW = 0, GF_EXEC_FUSED = 1 };

/* Runs photons first_id .. first_id + n - 1. exec GF_EXEC_FLOW runs the graph through the C++
 * Flow (partition + transforms + sink); GF_EXEC_FUSED carries each photon through the same
 * functors in one kernel (identical histories). Optional host outputs (NULL to skip):
 * h_event[n], h_scatter_count[n], h_weight[n], h_cos_exit[n], h_position[3n], h_direction[3n]
 * (per id, at the terminal event),
 * h_refl[hist_bins], h_trans[hist_bins] (summed exit weights), h_event_counts[5]. */
gf_status gf_run_photon(uint64_t seed, uint64_t first_id, uint64_t n, const gf_photon_params* h_params, int exec,
                        uint32_t chunk_capacity, uint32_t live_particles, uint32_t batch_chunks, uint32_t* h_event,
                        uint32_t* h_scatter_count, double* h_weight, double* h_cos_exit, double* h_position,
                        double* h_direction, double* h_refl, double* h_trans, uint64_t* h_event_counts,
                        gf_flow_stats* h_stats);

/* One path trace vertex (examples/photon_scattering/PhotonTypes.hpp:189-207 TraceVertexT): kind
 * 0 source, 1 scatter, 2 transmitted, 3 reflected, 4 absorbed, 5 capped; the completed scatters
 * (the scatter's own included); position and outgoing direction. */
typedef struct gf_trace_vertex {
    uint32_t kind;
    uint32_t scatter_count;
    double position[3];
    double direction[3];
} gf_trace_vertex;

/* gf_run_photon with the reference's bounded path trace (PhotonFunctors.hpp:201-234 TraceWriter,
 * recorded at the source, every scatter and the terminal event; PhotonScattering.hpp:49-82,
 * 158-174): photons with id < M = min(n, trace_photons) keep up to trace_vertices vertices each.
 * first_id must be 0 when trace_photons > 0 (GF_ERR_ARGUMENT otherwise, in both execution
 * forms); with trace_vertices = 0 no vertex fits, so every traced id reports truncated = 1.
 * Extra host outputs (NULL to skip):
 * h_trace_vertices[M * trace_vertices] (id-major; vertex j of id i at i * trace_vertices + j),
 * h_trace_counts[M] (vertices kept), h_trace_truncated[M] (1 when a vertex did not fit).
 * trace_photons = 0 runs exactly gf_run_photon. Histories are the same with or without a trace. */
gf_status gf_run_photon_traced(uint64_t seed, uint64_t first_id, uint64_t n, const gf_photon_params* h_params,
                               int exec, uint32_t chunk_capacity, uint32_t live_particles, uint32_t batch_chunks,
                               uint32_t* h_event, uint32_t* h_scatter_count, double* h_weight, double* h_cos_exit,
                               double* h_position, double* h_direction, double* h_refl, double* h_trans,
                               uint64_t* h_event_counts, gf_flow_stats* h_stats, uint32_t trace_photons,
                               uint32_t trace_vertices, gf_trace_vertex* h_trace_vertices, uint32_t* h_trace_counts,
                               uint32_t* h_trace_truncated);

/* Message of the last failed front-end call on this thread (empty if none). */
size_t gf_last_error(char* h_buf, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
