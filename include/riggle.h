/*
 * riggle.h — C ABI of riggle_b200, a B200 (sm_100a) implementation of the file-to-file
 * interval-sweep hot path of the `chuckle` crate (simondoesstuff/riggle).
 *
 * The ABI takes plain pointers and sizes only.  Each entry point names the reference interface it
 * replaces (file:line inside the reference crate).  Host buffers are owned by the caller; device
 * memory is owned by the handle that allocated it.  Every function returns an rgl_status; the
 * detail of the last failure on the calling thread is available from rgl_last_error().
 *
 * Semantics kept from the reference:
 *   - a query interval q and a database interval d overlap when
 *       q.start - layer_max_size(K) (saturating) <= d.start < q.end  and  d.end > q.start
 *     (src/sweep/query.rs:98-108, half-open intervals: touching ends do not overlap);
 *   - counts are u32 per (query row, database source) and wrap modulo 2^32 as the reference's
 *     release build does (src/matrix/dense.rs:42-45);
 *   - the reference's f32 "overlap bins" (src/sweep/query.rs:111-113) are returned as exact u64
 *     base pairs; bins = bp / bin_size.
 */
#ifndef RIGGLE_B200_H
#define RIGGLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------ */
/* Status codes.  Mirrors QueryError (src/tasks/query/mod.rs:26-38), LayerError                 */
/* (src/io/layer.rs:11-23), MetaError (src/io/meta.rs:9-15), BedParseError                      */
/* (src/io/parse.rs:22-38) and AddError (src/tasks/build.rs:18-32), plus device conditions.     */
/* ------------------------------------------------------------------------------------------ */
typedef enum rgl_status {
    RGL_OK = 0,
    RGL_ERR_INVALID_ARGUMENT = 1,
    RGL_ERR_IO = 2,                          /* QueryError::Io, LayerError::Io, MetaError::Io */
    RGL_ERR_BED_INVALID_FORMAT = 3,          /* BedParseError::InvalidFormat */
    RGL_ERR_BED_INVALID_START = 4,           /* BedParseError::InvalidStart */
    RGL_ERR_BED_INVALID_END = 5,             /* BedParseError::InvalidEnd */
    RGL_ERR_BED_INVALID_RANGE = 6,           /* BedParseError::InvalidRange (start >= end) */
    RGL_ERR_META_JSON = 7,                   /* MetaError::Json */
    RGL_ERR_LAYER_INVALID_POSITION_SIZE = 8, /* LayerError::InvalidPositionSize */
    RGL_ERR_LAYER_INVALID_SID_SIZE = 9,      /* LayerError::InvalidSidSize */
    RGL_ERR_LAYER_SID_SIZE_MISMATCH = 10,    /* LayerError::SidSizeMismatch */
    RGL_ERR_LAYER_INVALID_INDEX_SIZE = 11,   /* LayerError::InvalidIndexSize */
    RGL_ERR_DATABASE_NOT_FOUND = 12,         /* QueryError::DatabaseNotFound */
    RGL_ERR_INPUT_NOT_FOUND = 13,            /* AddError::InputNotFound */
    RGL_ERR_NO_BED_FILES = 14,               /* AddError::NoBedFiles */
    RGL_ERR_OOM = 15,                        /* device allocation failed / admission refused */
    RGL_ERR_TIMEOUT = 16,                    /* a bounded device wait gave up */
    RGL_ERR_DEVICE = 17,                     /* CUDA runtime error */
    RGL_ERR_INDEX_INVARIANT = 18,            /* layer unsorted, or a source id >= num_sources */
    RGL_ERR_NO_DEVICE = 19,                  /* no CUDA device visible */
    RGL_ERR_UNSUPPORTED = 20
} rgl_status;

const char* rgl_status_str(int status);
/* Detail of the last failure on this thread ("" when none). */
const char* rgl_last_error(void);
/* ABI version: major*10000 + minor*100 + patch. */
int rgl_version(void);

/* Layout of the public structs below as compiled into this library (no counterpart in the
 * reference; it lets a binding in another language check its declarations against the ABI).
 * rgl_abi_struct_name(i) names struct i (NULL past the last).  rgl_abi_layout fills sizeof,
 * alignof and the field count of the named struct, and for the first `capacity` fields in
 * declaration order their names, offsets and sizes (any output may be NULL). */
const char* rgl_abi_struct_name(uint32_t i);
int rgl_abi_layout(const char* name, uint64_t* size, uint64_t* align, uint32_t* num_fields,
                   const char** field_names, uint64_t* offsets, uint64_t* sizes, uint32_t capacity);

/* ------------------------------------------------------------------------------------------ */
/* Layer configuration — LayerConfig (src/io/meta.rs:23-90).  Pure host functions.             */
/* ------------------------------------------------------------------------------------------ */
/* LayerConfig::layer_for_size (src/io/meta.rs:33-58) */
uint32_t rgl_layer_for_size(uint32_t min_size, uint32_t growth_factor, uint32_t size);
/* LayerConfig::layer_max_size (src/io/meta.rs:64-73) */
uint32_t rgl_layer_max_size(uint32_t min_size, uint32_t growth_factor, uint32_t layer);
/* LayerConfig::tile_size (src/io/meta.rs:79-81) */
uint32_t rgl_tile_size(uint32_t min_size, uint32_t growth_factor, uint32_t layer);

/* Interval (src/core/mod.rs:11-17): 12-byte repr(C) {start, end, sid}. */
typedef struct rgl_interval {
    uint32_t start;
    uint32_t end;
    uint32_t sid;
} rgl_interval;

/* ------------------------------------------------------------------------------------------ */
/* Device-resident database index.                                                              */
/* ------------------------------------------------------------------------------------------ */
typedef struct rgl_index rgl_index;

/* One (shard, layer) in the reference's on-disk layout (src/io/layer.rs:31-47):
 * pos = layer_K.pos, `count` (start, end) u32 pairs sorted by start; sid = layer_K.sid. */
typedef struct rgl_layer_desc {
    uint32_t shard;
    uint32_t layer;
    uint64_t count;
    const uint32_t* pos;
    const uint32_t* sid;
} rgl_layer_desc;

typedef struct rgl_index_desc {
    uint32_t min_size;      /* LayerConfig.min_size (default 128) */
    uint32_t growth_factor; /* LayerConfig.growth_factor (default 4) */
    uint32_t num_sources;   /* Meta::num_sources (src/io/meta.rs:142-144) = matrix columns */
    uint32_t num_shards;
    const char* const* shard_names; /* may be NULL: shards named by their index */
    const char* const* source_names; /* may be NULL */
    uint32_t num_layers;            /* number of entries in `layers` */
    const rgl_layer_desc* layers;
} rgl_index_desc;

typedef struct rgl_index_info {
    uint32_t num_sources;
    uint32_t num_shards;
    uint32_t num_layer_slots; /* highest layer index + 1 */
    uint32_t num_layers;      /* non-empty (shard, layer) pairs */
    uint64_t num_intervals;
    uint64_t device_bytes;
    int device;
} rgl_index_info;

/* Opens `db_dir` written by the reference's `add` (src/tasks/build.rs:86-128): meta.json
 * (src/io/meta.rs:124-127) and shards/<shard>/layer_K.{pos,sid,idx} (src/io/layer.rs:51-78,
 * src/io/jump.rs:27-44), with the reference's size checks, and uploads the layers to HBM.
 * Replaces Meta::load + MappedLayer::open + MappedJumpTable::open in query_database
 * (src/tasks/query/mod.rs:124-129, 205-233). */
int rgl_index_open(const char* db_dir, int device, rgl_index** out);
/* Same from caller-owned host arrays (copied to HBM). */
int rgl_index_open_mem(const rgl_index_desc* desc, int device, rgl_index** out);
int rgl_index_close(rgl_index* index);
int rgl_index_get_info(const rgl_index* index, rgl_index_info* out);
/* Shard id for a name (RGL_ERR_INVALID_ARGUMENT when absent, as the reference skips shards not in
 * meta.shards: src/tasks/query/mod.rs:194-196). */
int rgl_index_shard_id(const rgl_index* index, const char* name, uint32_t* out_id);
const char* rgl_index_shard_name(const rgl_index* index, uint32_t shard);
const char* rgl_index_source_name(const rgl_index* index, uint32_t sid);
/* Column shard of an index (multi-GPU partition by database file, no counterpart in the reference):
 * a new index on the same device holding only the intervals with sid in [sid_lo, sid_hi), sids
 * rebased to 0, every layer still sorted by start.  Query results of the shard are the columns
 * [sid_lo, sid_hi) of the full index's results. */
int rgl_index_select_columns(const rgl_index* index, uint32_t sid_lo, uint32_t sid_hi, rgl_index** out);
/* add_to_database (src/tasks/build.rs:86-276) on the device: the BED files of input_path (*.bed,
 * *.bed.gz sorted by path, or one such file; every file gets the next D_SID, empty files included)
 * are parsed on `threads` host threads, bucketed by (shard, layer_for_size), sorted by start on the
 * device (equal starts keep file and line order) and merged into `base`'s layers (NULL: a new
 * index with layer config min_size / growth_factor) with new elements first on equal starts, as
 * the reference's reverse co-merge (extend_layer, src/io/layer.rs:129-199) orders them.  The result
 * is a new index on base's device (or `device`); base is unchanged.  RGL_ERR_INPUT_NOT_FOUND /
 * RGL_ERR_NO_BED_FILES as AddError. */
int rgl_index_add_beds(const rgl_index* base, const char* input_path, uint32_t min_size, uint32_t growth_factor,
                       uint32_t threads, int device, rgl_index** out);
/* Writes an index as a database directory in the reference's layout (meta.json and
 * shards/<shard>/layer_K.{pos,sid,idx}; the .idx is build_jump_table of the layer,
 * src/io/jump.rs:66-115), readable by rgl_index_open and by the reference's query. */
int rgl_index_write(const rgl_index* index, const char* db_dir);
/* Number of intervals of (shard, layer) (0 when absent). */
uint64_t rgl_index_layer_count(const rgl_index* index, uint32_t shard, uint32_t layer);
/* Copies one (shard, layer) back to host arrays of its count (2*count pos words, count sids). */
int rgl_index_export_layer(const rgl_index* index, uint32_t shard, uint32_t layer, uint32_t* pos, uint32_t* sid);

/* ------------------------------------------------------------------------------------------ */
/* Query contexts and the sweep.                                                                 */
/* ------------------------------------------------------------------------------------------ */
typedef struct rgl_context rgl_context;

/* A context binds one index to one CUDA stream and owns a reusable device workspace (grown on
 * demand, never shrunk).  `stream` is a cudaStream_t or NULL (the context creates its own). */
int rgl_context_create(rgl_index* index, void* stream, rgl_context** out);
int rgl_context_destroy(rgl_context* ctx);
/* Pre-sizes the workspace for batches of up to max_intervals query intervals and max_rows rows,
 * so later calls allocate nothing. */
int rgl_context_reserve(rgl_context* ctx, uint64_t max_intervals, uint32_t max_rows);
void* rgl_context_stream(rgl_context* ctx);

/* Queries of one shard: the reference's `shard_intervals[shard]` after parsing
 * (src/tasks/query/files.rs:40-111); `sid` of each interval is its query row (Q_SID).
 * `shard_name` selects the shard by name; when NULL, `shard_id` is used. */
typedef struct rgl_query_shard {
    const char* shard_name;
    uint32_t shard_id;
    uint64_t count;
    const rgl_interval* intervals;
} rgl_query_shard;

typedef struct rgl_query_batch {
    uint32_t num_rows; /* batch_len: query rows (src/tasks/query/mod.rs:184) */
    uint32_t num_shards;
    const rgl_query_shard* shards;
} rgl_query_batch;

/* Launch shape.  0 = default / autotuned. */
typedef struct rgl_query_opts {
    uint32_t chunk;       /* positions per work item (default 1024) */
    uint32_t ctas_per_sm; /* persistent CTAs per SM (default 8) */
    uint32_t block;       /* threads per CTA */
    uint32_t flags;       /* RGL_QF_* */
    uint32_t pair_ratio;  /* a candidate range is swept pair by pair when its candidates are at most
                             pair_ratio x its union size, else by rank differences (default 4) */
} rgl_query_opts;

#define RGL_QF_NO_OVERLAP 1u /* skip base-pair accumulation (counts only) */
#define RGL_QF_GLOBAL_TALLY 2u /* runs over several rows tally with atomics on the outputs instead of
                                  block-local histograms of each work item's row (for comparisons) */

typedef struct rgl_query_stats {
    uint64_t query_intervals;  /* intervals in the batch (on shards present in the index) */
    uint64_t db_swept;         /* DB intervals in the union of candidate ranges, all (shard, layer) */
    uint64_t rank_positions;   /* union elements swept by rank differences */
    uint64_t pair_candidates;  /* candidates swept pair by pair */
    uint64_t ranges;           /* merged candidate ranges */
    uint64_t work_items;       /* work items pulled by the sweep kernel */
    float sweep_ms;            /* sweep kernel time (CUDA events on the context stream) */
    float device_ms;           /* whole device pipeline incl. sort/partition (CUDA events) */
    uint32_t chunk, ctas_per_sm, block, kernel_launches;
} rgl_query_stats;

/* Replaces the counting path of query_database (src/tasks/query/mod.rs:182-307): the per-shard,
 * per-64-row-window, per-layer calls to query_sweep_windowed (src/sweep/query.rs:84-117) and the
 * window merge (add_submatrix_rows, src/matrix/dense.rs:75-86).  Host buffers: the batch is copied
 * to HBM, `counts` (num_rows x num_sources u32, row-major) and `overlap_bp` (same shape, u64; may
 * be NULL) are written on return.  Query intervals need start < end (the parser guarantees it,
 * src/io/parse.rs:94-100) and sid < num_rows. */
int rgl_query_counts(rgl_context* ctx, const rgl_query_batch* batch, const rgl_query_opts* opts, uint32_t* counts,
                     uint64_t* overlap_bp, rgl_query_stats* stats);

/* Device-resident variant: `d_intervals` (device, AoS) holds the shards back to back;
 * shard_offsets (host, num_shards+1) delimit them; shard_ids (host) name each block's shard.
 * d_counts / d_overlap_bp are device buffers.  Runs asynchronously on the context stream unless
 * stats is non-NULL (stats need one synchronisation). */
int rgl_query_counts_device(rgl_context* ctx, uint32_t num_rows, uint32_t num_shards, const uint32_t* shard_ids,
                            const uint64_t* shard_offsets, const rgl_interval* d_intervals,
                            const rgl_query_opts* opts, uint32_t* d_counts, uint64_t* d_overlap_bp,
                            rgl_query_stats* stats);

/* One overlapping pair of `--intervals` mode: IntervalHit (src/stats/mod.rs:4-15) with the query
 * file as its row, the database file as its sid and the chromosome as its shard id. */
typedef struct rgl_pair {
    uint32_t query_start, query_end;
    uint32_t db_start, db_end;
    uint32_t row;             /* query file (Q_SID) */
    uint32_t sid;             /* database source (D_SID) */
    uint32_t shard;           /* index shard (chromosome) */
    uint32_t intersection_bp; /* min(ends) - max(starts) */
} rgl_pair;

/* query_sweep_pairs (src/sweep/query.rs:11-41) driven as collect_interval_pairs
 * (src/tasks/query/intervals.rs:16-112): every overlapping (query interval, database interval) pair
 * of the batch with its exact intersection, in the order (layer, shard, row, query start, database
 * start); the reference's order differs only in the shard order (a HashMap's) and in placing rows
 * after start.  *out_count receives the number of pairs; with pairs == NULL nothing else is written,
 * else capacity must hold them all (RGL_ERR_INVALID_ARGUMENT otherwise).  Synchronous. */
int rgl_query_pairs(rgl_context* ctx, const rgl_query_batch* batch, uint64_t capacity, rgl_pair* pairs,
                    uint64_t* out_count);

/* ---- Batched form: many query files in one call -------------------------------------------------
 * Replaces query_database's loop over batches of query files (src/tasks/query/mod.rs:182-307) for a
 * whole set of files at once; the reference has no single entry point for it.  Block b holds
 * d_intervals[block_offsets[b] .. block_offsets[b+1]) on index shard block_shards[b]; blocks are laid
 * end to end (offsets non-decreasing).  Every interval's sid is its output row (query file).  With
 * block_rows given, all intervals of block b have sid == block_rows[b], which narrows the rows each
 * sub-batch touches; with NULL they may lie anywhere in [0, num_rows). */
typedef struct rgl_batch {
    uint32_t num_rows;
    uint32_t num_blocks;
    const uint32_t* block_shards;    /* host, num_blocks */
    const uint32_t* block_rows;      /* host, num_blocks, or NULL */
    const uint64_t* block_offsets;   /* host, num_blocks + 1 */
    const rgl_interval* d_intervals; /* device */
} rgl_batch;

typedef struct rgl_batch_opts {
    rgl_query_opts query; /* launch shape of every sub-batch (zeros: tuned shape or defaults) */
    uint64_t sub_batch;   /* query intervals per sub-batch, the unit of device workspace (0: 2^25) */
    uint32_t flags;       /* RGL_BF_* */
    uint32_t region_bits; /* work order of a sub-batch of several rows: each row's intervals on a shard
                             are cut into 2^region_bits-bp regions of their starts and the work is
                             laid out region by region, every row's work on a region together, so the
                             database intervals of a region are read from L2 by all rows after the
                             first.  0 or RGL_BATCH_NO_REGIONS: one segment per (shard, row) (the
                             default: measured against the 2e9-interval database the region order
                             gained nothing, the sweeps are not limited by DRAM traffic); else
                             16..31.  Results do not depend on it; the swept count (stats) grows by
                             the look-back windows that cross region boundaries. */
} rgl_batch_opts;

#define RGL_BATCH_NO_REGIONS 32u

#define RGL_BF_GRAPH 1u /* capture the batch as one CUDA graph and replay it while the batch (its block
                           tables, buffers and launch shape) is unchanged */
#define RGL_BF_TUNED 2u /* fill zero launch fields from the context's rgl_batch_autotune result */

typedef struct rgl_batch_stats {
    uint64_t query_intervals;  /* intervals in the batch */
    uint64_t db_swept;         /* per query file: the union of its candidate ranges, summed */
    uint64_t rank_positions;   /* union elements swept by rank differences */
    uint64_t pair_candidates;  /* candidates swept pair by pair */
    uint64_t ranges;           /* merged candidate ranges */
    uint32_t sub_batches;      /* pipeline runs */
    uint32_t kernel_launches;  /* kernels of this library launched (CUB's not counted) */
    uint32_t graph_nodes;      /* nodes of the captured graph (0 without RGL_BF_GRAPH) */
    uint32_t graph_replayed;   /* 1: an identical earlier batch's graph was launched again */
    float device_ms;           /* CUDA events around the whole batch on the context stream */
    uint32_t chunk, ctas_per_sm, pair_ratio;
} rgl_batch_stats;

/* Zeroes d_counts (num_rows x D) and d_overlap_bp, then accumulates every sub-batch into them.
 * Asynchronous on the context stream unless stats is non-NULL; errors in the intervals are then
 * reported by rgl_context_check.  The first call with RGL_BF_GRAPH sizes the workspace, captures and
 * launches; later identical calls launch the cached graph without host work per sub-batch. */
int rgl_query_batch_device(rgl_context* ctx, const rgl_batch* batch, const rgl_batch_opts* opts,
                           uint32_t* d_counts, uint64_t* d_overlap_bp, rgl_batch_stats* stats);

/* The batched form with the intervals in host memory (page-locked for full speed; batch->d_intervals
 * is ignored): sub-batch k + 1 is copied to the device on a second stream while sub-batch k is swept.
 * counts / overlap_bp are host buffers (num_rows x D).  Synchronous; not graph-captured. */
int rgl_query_batch_host(rgl_context* ctx, const rgl_batch* batch, const rgl_interval* h_intervals,
                         const rgl_batch_opts* opts, uint32_t* counts, uint64_t* overlap_bp,
                         rgl_batch_stats* stats);

typedef struct rgl_tune_trial {
    uint32_t chunk, ctas_per_sm, pair_ratio;
    float sweep_ms; /* best of two runs of the sweep kernels of the largest sub-batch */
} rgl_tune_trial;

/* Autotuner: times the sweep kernels of the batch's largest sub-batch for pair_ratio in {1,2,4,8}
 * at the default shape, then for work-item size {512..8192} x CTAs per SM {2,3,4,6,8}; stores the
 * fastest shape in the context (used by RGL_BF_TUNED) and returns it in *best.  trials (optional)
 * receives up to max_trials measurements. */
int rgl_batch_autotune(rgl_context* ctx, const rgl_batch* batch, uint64_t sub_batch, rgl_query_opts* best,
                       rgl_tune_trial* trials, uint32_t max_trials, uint32_t* num_trials);

/* ------------------------------------------------------------------------------------------ */
/* Sliding-window moment store and analytic p-values.                                           */
/* ------------------------------------------------------------------------------------------ */
/* compact_index (src/fourier/moments.rs:58-66): store slot of block size l >= 1. */
uint64_t rgl_compact_index(uint64_t l);
/* The L values a chromosome of n_bins bins stores, in store order (src/fourier/moments.rs:215-247);
 * returns their number, writes min(number, capacity). */
uint64_t rgl_moment_grid(uint64_t n_bins, uint64_t* out_l, uint64_t capacity);
/* build_query_chrom_data (src/fourier/moments.rs:138-177) for one query file's intervals on one
 * chromosome: lengths in bins grouped by l_int = max(ceil(len / bin_size), 1), ascending, with
 * sum_scale = sum(l / l_int), sum_scale2 = sum((l / l_int)^2) and count. */
int rgl_query_chrom_groups(const rgl_interval* intervals, uint64_t n, uint32_t bin_size, uint64_t* l_int,
                           double* sum_scale, double* sum_scale2, uint64_t* count, uint64_t capacity,
                           uint64_t* out_groups);

/* Device-resident moment store: one (mean, var) f32 table per (source, chromosome), as the
 * reference's momentmap keeps them (src/io/momentstore.rs:22-34; the rkyv file format itself is
 * not read).  n_bins[c] = ceil(chromosome size / bin size) fixes each chromosome's L grid. */
typedef struct rgl_moments rgl_moments;
int rgl_moments_create(int device, uint32_t num_sources, uint32_t num_chroms, const uint64_t* n_bins,
                       rgl_moments** out);
int rgl_moments_destroy(rgl_moments* m);
/* Entries of a full table for the chromosome (the L grid size). */
uint64_t rgl_moments_slots(const rgl_moments* m, uint32_t chrom);
/* MomentStoreBuilder::insert for one (source, chromosome) (src/io/momentstore.rs:134-154):
 * `entries` (mean, var) f32 pairs in store order; 0 entries = no table. */
int rgl_moments_set(rgl_moments* m, uint32_t sid, uint32_t chrom, const float* mean_var, uint64_t entries);
int rgl_moments_get(const rgl_moments* m, uint32_t sid, uint32_t chrom, float* mean_var, uint64_t capacity,
                    uint64_t* out_entries);

/* build_depth_signal (src/fourier/depth.rs:109-204) on the device: the f32 coverage of one source on
 * one chromosome of n_bins bins, bit for bit the reference's (same impulse and prefix-sum order).
 * Intervals in the source file's order; g_out holds n_bins floats. */
int rgl_depth_signal(int device, const rgl_interval* intervals, uint64_t n, uint64_t n_bins, uint32_t bin_size,
                     float* g_out);
/* Allocation-free depth signal (no counterpart in the reference).  For callers that cannot
 * allocate device memory during the call: code recording a CUDA graph (cudaMalloc is not a
 * capturable operation), hosts that route every device allocation through their own arena, and
 * latency-critical loops that cannot take cudaMalloc's implicit synchronisation.  Same result as
 * rgl_depth_signal, from device-resident intervals into d_g (n_bins floats, device), enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) without synchronising.  Its scratch is a
 * static device array of RGL_NOALLOC_SCRATCH_BYTES (17 MiB) that every GPU loading the library
 * holds until exit; inputs above RGL_NOALLOC_MAX_INTERVALS intervals or RGL_NOALLOC_MAX_BINS bins
 * are rejected with RGL_ERR_INVALID_ARGUMENT, and so are a d_g that is not 16-byte aligned (it is
 * read and written as float4) and d_intervals that are not 4-byte aligned.  The first call on a
 * device looks up the array's device address (make it before any stream capture); the address is
 * looked up again when the device's context has been replaced since (cudaDeviceReset), so make the
 * first call after such a reset before any capture too.  All calls share the array: calls that may
 * overlap on the GPU (different streams, or threads) race and must be serialised by the caller. */
#define RGL_NOALLOC_MAX_INTERVALS 65536u
#define RGL_NOALLOC_MAX_BINS 4194304u
#define RGL_NOALLOC_SCRATCH_BYTES (17u << 20)
int rgl_depth_signal_noalloc(int device, const rgl_interval* d_intervals, uint64_t n, uint64_t n_bins,
                             uint32_t bin_size, float* d_g, void* stream);
/* build_chrom_moments (src/fourier/moments.rs:129-132, 192-254) on the device for (sid, chrom) of the
 * store: depth signal, FP64 Stockham-FFT autocorrelation of the centred signal and double-double
 * prefix sums, FP64 window mean / variance for the chromosome's L grid, stored as f32.
 * mean_out / var_out (optional, host, grid length) receive the FP64 values. */
int rgl_moments_build(rgl_moments* m, uint32_t sid, uint32_t chrom, const rgl_interval* intervals, uint64_t n,
                      uint32_t bin_size, double* mean_out, double* var_out);
/* rgl_moments_build with a choice of arithmetic for the FFT autocorrelation and the prefix sums
 * (the reference computes them in f64 with rustfft, src/fourier/moments.rs:421-466):
 *   RGL_MOM_FP64  - FP64 Stockham FFT and double-double prefix sums (rgl_moments_build);
 *   RGL_MOM_FP32C - compensated FP32: the centred signal scaled by a power of two per chromosome,
 *                   a float-float (two-sum / FMA two-product) Stockham FFT, power spectrum and
 *                   prefix sums, FP64 only in the final per-L reduction and the variance
 *                   subtraction.  About 48 significant bits per value.
 * The depth signal is the reference's f32 signal bit for bit in both. */
#define RGL_MOM_FP64 0u
#define RGL_MOM_FP32C 1u
int rgl_moments_build_ex(rgl_moments* m, uint32_t sid, uint32_t chrom, const rgl_interval* intervals, uint64_t n,
                         uint32_t bin_size, uint32_t precision, double* mean_out, double* var_out);

/* Query length groups of a batch: row q owns groups [row_group_offsets[q], row_group_offsets[q+1]),
 * each on chromosome group_chrom[g] of the moment store. */
typedef struct rgl_pvalue_batch {
    uint32_t num_rows;
    const uint64_t* row_group_offsets;
    const uint32_t* group_chrom;
    const uint64_t* group_l_int;
    const double* group_sum_scale;
    const double* group_sum_scale2;
    const uint64_t* group_count;
} rgl_pvalue_batch;

#define RGL_PV_EMITTED 1u /* count > 0 and a chromosome shared with moments (the reference emits it) */
#define RGL_PV_HAS_LLR 2u /* the NB / Poisson LLR exists (PValueResult.llr is Some) */

/* compute_analytic_pvalues + compute_analytic_stats (src/tasks/query/pvalues.rs:22-77,
 * src/fourier/stats.rs:34-126) for every (row, source) cell with a non-zero count, in FP64.
 * observed = overlap_bp / bin_size (exact; the reference sums f32 bins).  Outputs are dense
 * num_rows x num_sources host arrays: p, llr, log_p (ln p evaluated without underflow; may be
 * NULL) and flags (RGL_PV_*).  Cells not emitted hold p = 1, llr = 0, flags = 0. */
int rgl_query_pvalues(rgl_moments* m, const rgl_pvalue_batch* batch, uint32_t bin_size, const uint32_t* counts,
                      const uint64_t* overlap_bp, double* p, double* llr, double* log_p, uint8_t* flags);

/* The stats stage of the batched form, all on the device: compute_analytic_pvalues
 * (src/tasks/query/pvalues.rs:22-77) for every (row, source) cell of a batch whose counts and overlap
 * are in device memory (the outputs of rgl_query_batch_device), with the query length groups
 * (build_query_chrom_data, src/fourier/moments.rs:138-177) built on the device from the batch's own
 * intervals.  The group sums come from exact integer sums of lengths and squared lengths (one
 * rounding each; the reference rounds sequentially, ~1e-15 relative apart).  shard_chrom maps index
 * shard -> moment-store chromosome (UINT32_MAX: none); batch->block_rows is required.  Outputs are
 * device arrays of num_rows x D (d_log_p may be NULL), written asynchronously on the context
 * stream; *out_groups (optional, synchronises) receives the number of groups. */
int rgl_batch_pvalues_device(rgl_context* ctx, rgl_moments* moments, const rgl_batch* batch,
                             const uint32_t* shard_chrom, uint32_t num_shards, uint32_t bin_size,
                             const uint32_t* d_counts, const uint64_t* d_overlap_bp, double* d_p, double* d_llr,
                             double* d_log_p, uint8_t* d_flags, uint64_t* out_groups);

/* The query length groups that rgl_batch_pvalues_device builds on the device from the batch's own
 * intervals (build_query_chrom_data, src/fourier/moments.rs:138-177, for every (row, chromosome)),
 * copied to host memory: row q owns groups [row_group_offsets[q], row_group_offsets[q+1])
 * (num_rows + 1 entries), ascending by (chromosome, l_int).  Groups whose l_int reaches the
 * chromosome's n_bins are not materialised: the reference's store lookup returns None for them
 * (src/io/momentstore.rs:66-79).  *out_groups receives the count; with every group array NULL only
 * the offsets are written, else capacity must hold all groups.  Synchronous. */
int rgl_batch_query_groups(rgl_context* ctx, rgl_moments* moments, const rgl_batch* batch,
                           const uint32_t* shard_chrom, uint32_t num_shards, uint32_t bin_size,
                           uint64_t* row_group_offsets, uint32_t* group_chrom, uint64_t* group_l_int,
                           double* group_sum_scale, double* group_sum_scale2, uint64_t* group_count,
                           uint64_t capacity, uint64_t* out_groups);

/* ------------------------------------------------------------------------------------------ */
/* Results: sparse counts and the reference's JSON output.                                       */
/* ------------------------------------------------------------------------------------------ */
/* K9 on the device: the non-zero cells of a dense num_rows x num_sources count matrix (device,
 * e.g. rgl_query_batch_device's output) as CSR in (row, column) order, which is how query_database
 * collects all_entries and builds its CsMat (src/tasks/query/mod.rs:288-307,
 * build_csr_from_sorted_entries src/tasks/query/sweep.rs:4-23).  d_indptr (num_rows + 1, device)
 * always receives the row pointers and *out_nnz the entry count (synchronises).  With d_indices
 * non-NULL the column indices, and the counts (d_values) and overlap base pairs (d_bp_values, which
 * needs d_overlap_bp) where given, are written for the first `capacity` entries;
 * RGL_ERR_INVALID_ARGUMENT when nnz exceeds capacity.  Runs on the context's stream. */
int rgl_dense_to_csr_device(rgl_context* ctx, uint32_t num_rows, uint32_t num_sources, const uint32_t* d_counts,
                            const uint64_t* d_overlap_bp, uint64_t* d_indptr, uint32_t* d_indices,
                            uint32_t* d_values, uint64_t* d_bp_values, uint64_t capacity, uint64_t* out_nnz);

/* The StatsOutput JSON of `chuckle query` (src/main.rs:141-204; StatResult, src/stats/mod.rs:30-60,
 * serde_json::to_string_pretty), byte for byte: one result per CSR entry (host arrays, e.g. copied
 * from rgl_dense_to_csr_device) with its query / database names and overlap count.  With p_value
 * non-NULL (stats mode; observed_bins, p_value, llr and flags are dense num_rows x num_sources host
 * arrays as rgl_query_pvalues writes them) only cells flagged RGL_PV_EMITTED are written, with
 * observed_bins, p_value and llr (when RGL_PV_HAS_LLR), sorted by ascending p-value (ties in
 * (query, database) order; the reference's follow a HashMap); without, every entry, sorted by
 * descending overlap count (stable, as the reference).  *out_len receives the byte length; with out
 * NULL nothing else is written, else capacity must hold it (no terminating NUL is added). */
int rgl_format_stats_json(uint32_t num_rows, uint32_t num_sources, const char* const* query_names,
                          const char* const* db_names, const uint64_t* indptr, const uint32_t* indices,
                          const uint32_t* counts, const double* observed_bins, const double* p_value,
                          const double* llr, const uint8_t* flags, char* out, uint64_t capacity,
                          uint64_t* out_len);
/* The IntervalsOutput JSON of `chuckle query --intervals` (IntervalHit, src/stats/mod.rs:4-27): one
 * hit per rgl_pair in the given order, names taken by row, sid and shard. */
int rgl_format_intervals_json(const rgl_pair* pairs, uint64_t n, uint32_t num_rows, uint32_t num_sources,
                              uint32_t num_shards, const char* const* query_names, const char* const* db_names,
                              const char* const* shard_names, char* out, uint64_t capacity, uint64_t* out_len);

/* ------------------------------------------------------------------------------------------ */
/* Seeded synthetic workloads (no counterpart in the reference; used by tests and benchmarks).  */
/* SplitMix64 counter streams (Steele, Lea & Flood 2014) drive identical host and device        */
/* generators; lengths come from a host-built 65537-point quantile table.                       */
/* ------------------------------------------------------------------------------------------ */
typedef struct rgl_synth_spec {
    uint64_t seed;          /* per-dataset seed (files use seed + file index) */
    uint32_t num_chroms;    /* chromosome count (names chr1..chr22, chrX, chrY for 24) */
    const uint32_t* chrom_len;
    uint32_t num_files;
    const uint64_t* file_sizes; /* intervals per file */
    double broad_fraction;      /* share of intervals with log-uniform[10k,1M] lengths */
    double hotspot_fraction;    /* share placed in 1 Mbp hot spots */
    uint32_t num_hotspots;      /* hot spots per file */
    uint32_t sid_base;          /* sid of file 0 */
} rgl_synth_spec;

/* Chromosome lengths uniform in [50M, 250M] from `seed`. */
int rgl_synth_chrom_lengths(uint64_t seed, uint32_t num_chroms, uint32_t* out);
/* Rank-size Zipf file sizes clamp(round(C r^-s), lo, hi) with C chosen so the sum is ~target. */
int rgl_synth_zipf_sizes(uint32_t num_files, double s, uint64_t lo, uint64_t hi, uint64_t target, uint64_t* out);
/* Log-uniform file sizes in [lo, hi]. */
int rgl_synth_loguniform_sizes(uint64_t seed, uint32_t num_files, uint64_t lo, uint64_t hi, uint64_t* out);
/* Intervals of file f split over chromosomes (proportional split, largest remainder). */
int rgl_synth_file_chrom_counts(const rgl_synth_spec* spec, uint32_t file, uint64_t* out_per_chrom);
/* Host generation of one (file, chrom) block, sorted by (start, end); sid = sid_base + file. */
int rgl_synth_block_host(const rgl_synth_spec* spec, uint32_t file, uint32_t chrom, rgl_interval* out,
                         uint64_t capacity, uint64_t* out_count);
/* Host generation of every file's intervals on one chromosome, bucketed into layers like the
 * reference's add (src/tasks/build.rs:190-211): pos/sid are sorted by (layer, start) and
 * layer_counts[K] (K < max_layers) gives each layer's length.  Call with pos = sid = NULL to get
 * *out_total first. */
int rgl_synth_chrom_layers_host(const rgl_synth_spec* spec, uint32_t chrom, uint32_t min_size, uint32_t growth_factor,
                                uint64_t* layer_counts, uint32_t max_layers, uint32_t* pos, uint32_t* sid,
                                uint64_t capacity, uint64_t* out_total);
/* Builds an index in HBM directly from a spec (generation, bucketing by (shard, layer) and sort by
 * start all on the device).  Same content as bucketing the host blocks. */
int rgl_index_synth(const rgl_synth_spec* spec, uint32_t min_size, uint32_t growth_factor, int device,
                    rgl_index** out);
/* The same for files [file_lo, file_hi) only (each with its global stream; sid = sid_base + f -
 * file_lo): one GPU's column shard of a database too large for one GPU. */
int rgl_index_synth_columns(const rgl_synth_spec* spec, uint32_t min_size, uint32_t growth_factor, uint32_t file_lo,
                            uint32_t file_hi, int device, rgl_index** out);
/* File-major layout of a query batch drawn from a spec: block f * num_chroms + c holds the intervals
 * of (file f, chromosome c), sized as rgl_synth_file_chrom_counts.  block_offsets receives
 * num_files * num_chroms + 1 entries; block_shards (= c) and block_rows (= f) are optional. */
int rgl_synth_batch_layout(const rgl_synth_spec* spec, uint64_t* block_offsets, uint32_t* block_shards,
                           uint32_t* block_rows);
/* Generates that batch into device memory: block (f, c) holds the intervals rgl_synth_block_host
 * returns for (f, c), in generation order (unsorted), sid = sid_base + f.  Synchronises `stream`. */
int rgl_synth_batch_device(const rgl_synth_spec* spec, int device, const uint64_t* block_offsets,
                           rgl_interval* d_out, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* BED ingest: parse_bed_file (src/io/parse.rs:47-141) and parse_file_batch / enumerate_query_files */
/* (src/tasks/query/files.rs:25-111), native and multi-threaded on the host.                    */
/* ------------------------------------------------------------------------------------------ */
typedef struct rgl_bed_batch rgl_bed_batch;

/* The BED files under query_path sorted by path (*.bed, *.bed.gz), or query_path itself; parsed on
 * `threads` host threads (0: all cores).  Files without intervals are dropped and the rest numbered
 * 0.. in path order (compact Q_SIDs, written into every interval's sid).  Errors: RGL_ERR_INPUT_NOT_FOUND,
 * RGL_ERR_IO, RGL_ERR_BED_INVALID_FORMAT / _RANGE with the file and 1-based line in rgl_last_error. */
int rgl_bed_batch_load(const char* query_path, uint32_t threads, rgl_bed_batch** out);
/* parse_bed_string (src/io/parse.rs:143-160): one row from text, kept even when empty. */
int rgl_bed_parse_string(const char* text, uint64_t len, uint32_t sid, rgl_bed_batch** out);
uint32_t rgl_bed_batch_rows(const rgl_bed_batch* batch);
const char* rgl_bed_batch_row_name(const rgl_bed_batch* batch, uint32_t row);  /* the file name */
uint64_t rgl_bed_batch_row_count(const rgl_bed_batch* batch, uint32_t row);
uint32_t rgl_bed_batch_row_shards(const rgl_bed_batch* batch, uint32_t row);
/* Shard k of a row (first-appearance order): its name and intervals (file order). */
int rgl_bed_batch_block(const rgl_bed_batch* batch, uint32_t row, uint32_t k, const char** shard,
                        const rgl_interval** intervals, uint64_t* count);
/* query_database's counting path over a parsed batch: rgl_query_counts with one shard entry per
 * (row, shard) block; shards absent from the index are skipped (src/tasks/query/mod.rs:194-196). */
int rgl_bed_batch_query(rgl_context* ctx, const rgl_bed_batch* batch, const rgl_query_opts* opts, uint32_t* counts,
                        uint64_t* overlap_bp, rgl_query_stats* stats);
int rgl_bed_batch_free(rgl_bed_batch* batch);

/* ------------------------------------------------------------------------------------------ */
/* Request server (no counterpart in the reference, whose query_database answers one set of     */
/* files per process run).  The index stays resident; query files arrive one at a time and are   */
/* batched as they come: each worker owns a query context on its own stream and, whenever it is  */
/* idle, takes the oldest pending requests (up to max_batch_requests and batch_intervals) as one */
/* batch, so requests that arrive while others are on the GPU overlap with them on the device.   */
/* ------------------------------------------------------------------------------------------ */
typedef struct rgl_server rgl_server;

/* Free device memory as the server sees it when it forms a batch (bytes); the default asks the
 * CUDA runtime (cudaMemGetInfo).  Called with the server's queue lock held, from worker threads. */
typedef uint64_t (*rgl_free_memory_fn)(void* user);

typedef struct rgl_server_opts {
    uint32_t workers;               /* batches in flight at once (default 3; fewer when HBM is short) */
    uint32_t max_batch_requests;    /* requests per batch (default 256; 1 = one query file per launch) */
    uint64_t batch_intervals;       /* intervals per batch, also the largest admissible request (default 2^23) */
    uint64_t hbm_reserve_bytes;     /* device memory every admission leaves free (default 4 GiB) */
    uint64_t max_pending_intervals; /* host queue bound: submit refuses beyond it (default 2^28) */
    rgl_query_opts query;           /* launch shape (zeros: defaults); RGL_QF_NO_OVERLAP */
    uint64_t initial_intervals;     /* workspace each worker reserves at creation (default
                                       batch_intervals: no growth while serving); batches beyond it
                                       grow the workspace when free device memory admits them (a
                                       growth reallocates, which synchronises the device) */
    rgl_free_memory_fn free_memory; /* NULL: cudaMemGetInfo */
    void* free_memory_user;
    rgl_moments* moments;           /* non-NULL: every request also gets its p-values (stats stage) */
    const uint32_t* shard_chrom;    /* index shard -> moment-store chromosome (UINT32_MAX: none) */
    uint32_t num_shard_chrom;
    uint32_t bin_size;              /* bin of the moment store (default 100) */
} rgl_server_opts;

/* One query file.  The server copies the block tables at submit; `intervals` (page-locked for
 * asynchronous copies) must stay valid until the request completes; counts / overlap_bp (D entries
 * each, overlap_bp may be NULL) are written when it completes, and with a moment store p_value,
 * llr, log_p and flags (D entries each, any may be NULL; as rgl_query_pvalues writes them for one
 * row).  Interval sids are ignored. */
typedef struct rgl_request {
    uint32_t num_blocks;
    const uint32_t* block_shards;  /* index shard of each block */
    const uint64_t* block_offsets; /* num_blocks + 1 element offsets into intervals */
    const rgl_interval* intervals;
    uint32_t* counts;
    uint64_t* overlap_bp;
    double* p_value;
    double* llr;
    double* log_p;
    uint8_t* flags;
} rgl_request;

typedef struct rgl_request_info {
    int status;               /* rgl_status of this request */
    uint32_t batch_requests;  /* requests in the batch it ran in */
    uint64_t batch_intervals; /* intervals in that batch */
    uint64_t intervals;       /* this request's intervals */
    double submit_s, start_s, done_s; /* steady-clock seconds since the server was created */
} rgl_request_info;

typedef struct rgl_server_stats {
    uint64_t submitted, completed, failed, batches, intervals;
    uint32_t workers;           /* workers admitted by free HBM */
    uint32_t pending;           /* requests waiting now */
    double mean_batch_requests;
    double p50_ms, p99_ms, p999_ms, max_ms, mean_ms; /* submit -> results in host memory */
    double first_submit_s, last_done_s;
    double worker_bytes;        /* device memory of the first worker at creation */
    uint64_t memory_limited;    /* batches closed early because free device memory admitted no more */
    uint64_t refused;           /* requests failed with RGL_ERR_OOM: larger than free memory admits */
    uint64_t grown_bytes;       /* device memory the workers' workspaces grew by after creation */
} rgl_server_stats;

/* Creates the workers (each with its initial workspace while free device memory allows).  A worker
 * forms each batch from the oldest pending requests: a request joins when the batch stays within
 * max_batch_requests and batch_intervals and the device memory the batch would add to the worker's
 * workspace fits in the free memory (free_memory()) less hbm_reserve_bytes and less what other
 * workers have been promised; a request that does not fit even alone is failed with RGL_ERR_OOM.
 * free_memory() is called only for a batch that would grow the worker's buffers (a batch within
 * them needs no admission), and without the server's lock held, so a slow query (cudaMemGetInfo
 * can take tens of milliseconds on a busy node) delays neither submissions nor other workers.
 * Workers wait for their batches by polling with yields (a blocking synchronisation after 100 ms).
 * The server's moment store (optional) must outlive it. */
int rgl_server_create(rgl_index* index, const rgl_server_opts* opts, rgl_server** out);
/* Queues one request; RGL_ERR_INVALID_ARGUMENT for a bad block table or a request larger than
 * batch_intervals, RGL_ERR_OOM when the queue is full. */
int rgl_server_submit(rgl_server* server, const rgl_request* req, uint64_t* ticket);
/* Waits up to timeout_ms (0: poll) for a request; RGL_ERR_TIMEOUT while it is not done.  A completed
 * ticket is released by this call.  A batch that fails is retried request by request, so only the
 * request with invalid intervals fails. */
int rgl_server_wait(rgl_server* server, uint64_t ticket, uint32_t timeout_ms, rgl_request_info* info);
int rgl_server_get_stats(rgl_server* server, rgl_server_stats* out);
/* Clears the latency record and counters (between a warm-up and a measured run). */
int rgl_server_reset_stats(rgl_server* server);
/* Finishes the queued requests, stops the workers and frees everything. */
int rgl_server_destroy(rgl_server* server);

/* ------------------------------------------------------------------------------------------ */
/* Stream helpers, timing and pinned host memory (no counterpart in the reference).              */
/* ------------------------------------------------------------------------------------------ */
int rgl_context_sync(rgl_context* ctx);
/* Synchronises the context stream and reports a query error raised by the last asynchronous
 * rgl_query_counts_device call (invalid query intervals). */
int rgl_context_check(rgl_context* ctx);
/* When on, every sweep launch is bracketed by CUDA events on the context stream. */
int rgl_context_set_timing(rgl_context* ctx, int on);
/* Synchronises, returns the summed sweep-kernel time and launch count since the last call. */
int rgl_context_sweep_times(rgl_context* ctx, float* total_ms, uint32_t* launches);
/* Page-locked host buffers for fast host<->device copies. */
int rgl_host_alloc(uint64_t bytes, void** out);
int rgl_host_free(void* ptr);

#ifdef __cplusplus
}
#endif

#endif /* RIGGLE_B200_H */
