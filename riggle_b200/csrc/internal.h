// Internal declarations shared by the host and device translation units of libriggle_b200.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/riggle.h"

namespace rgl {

// ---- errors ------------------------------------------------------------------------------------
// Sets the thread-local detail string and returns `code`.
int fail(int code, const std::string& msg);
void clear_error();

#define RGL_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return ::rgl::fail(e_ == cudaErrorMemoryAllocation ? RGL_ERR_OOM : RGL_ERR_DEVICE,      \
                               std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

#define RGL_TRY(expr)                     \
    do {                                  \
        int s_ = (expr);                  \
        if (s_ != RGL_OK) return s_;      \
    } while (0)

// Makes `device` current for the scope and gives the calling thread its previous device back on
// exit, so an entry point leaves the caller's device selection as it found it.
struct DeviceScope {
    int prev = -1;
    int enter(int device) {
        RGL_CUDA(cudaGetDevice(&prev));
        RGL_CUDA(cudaSetDevice(device));
        return RGL_OK;
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// ---- layer configuration (src/io/meta.rs:33-81) ---------------------------------------------
uint32_t layer_for_size(uint32_t min_size, uint32_t gf, uint32_t size);
uint32_t layer_max_size(uint32_t min_size, uint32_t gf, uint32_t layer);
uint32_t tile_size(uint32_t min_size, uint32_t gf, uint32_t layer);

// ---- device index ------------------------------------------------------------------------------
// One non-empty (shard, layer).  `off` is the element offset of the layer in the index-wide pos
// (uint2) and sid (u32) arrays; offsets are multiples of 4 so every layer starts 16-byte aligned.
struct LayerDev {
    uint64_t off;
    uint64_t n;
    uint32_t max_size;  // layer_max_size(K): the look-back of the sweep
    uint32_t shard;
    uint32_t layer;
    uint32_t flags;  // LF_* bits from validation
    // bucket table (built by index_finalize): d_btab[boff + b] = #(start < b << bshift) for b < nb,
    // buckets of 2^bshift bp holding about one interval each; d_btab[boff + nb - 1] = n
    uint64_t boff;
    uint32_t bshift, nb;
};
enum : uint32_t { LF_UNSORTED = 1u, LF_BAD_SID = 2u, LF_EMPTY_IV = 4u, LF_OVERSIZE = 8u };

// A device allocation that grows on demand (never shrinks).
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);  // cudaMalloc (after cudaFree) when bytes > cap
    void release();
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

// Scratch of the batched stats stage (query length groups of a batch); one per concurrent caller.
struct StatsScratch {
    DevBuf key_a, key_b, len_a, len_b, ukey, agg, runs, groups, goff, tmp;
    DevBuf plan;  // block-local form: the sort's plan and order flags, run-head counts per tile
};

}  // namespace rgl

struct rgl_index {
    int device = 0;
    uint32_t min_size = 128, gf = 4, num_sources = 0, num_shards = 0, num_slots = 0;
    std::vector<std::string> shard_names;
    std::unordered_map<std::string, uint32_t> shard_ids;
    std::vector<std::string> source_names;
    std::vector<rgl::LayerDev> layers;  // host copy of the layer table
    std::vector<int32_t> slot;          // [shard * num_slots + K] -> layer index or -1
    uint64_t total = 0;                 // intervals
    uint64_t cap_elems = 0;             // allocated elements (with alignment padding)
    uint2* d_pos = nullptr;
    uint32_t* d_sid = nullptr;
    rgl::LayerDev* d_layers = nullptr;
    uint32_t* d_btab = nullptr;         // bucket tables of all layers
    int32_t* d_slot = nullptr;
    uint64_t device_bytes = 0;
    // one reference for the handle returned to the caller plus one per live context; the device
    // memory is released when the last reference goes (rgl_index_close may precede the contexts)
    std::atomic<int> refs{1};
};

namespace rgl {

// Allocates the device arrays of an index whose host-side layer table is filled (layers, slot,
// total computed from counts); assigns aligned offsets.
int index_alloc(rgl_index* idx);
// Uploads the layer tables and validates every layer on the device (sortedness, source ids,
// non-empty intervals, size class).  Fails with RGL_ERR_INDEX_INVARIANT on an unsorted layer or a
// source id >= num_sources.
int index_finalize(rgl_index* idx);
void index_free(rgl_index* idx);
void index_release(rgl_index* idx);

// ---- host IO (src/io) -------------------------------------------------------------------------
struct MetaInfo {
    std::unordered_map<uint32_t, std::string> sid_map;
    uint32_t min_size = 128, growth_factor = 4;
    std::vector<std::string> shards;
    uint64_t num_layers = 0;
};
int meta_load(const std::string& db_dir, MetaInfo* out);
int read_file(const std::string& path, std::vector<uint8_t>* out);
bool file_exists(const std::string& path);

// ---- synthetic generator (shared host/device arithmetic) ---------------------------------------
struct SynthTables {
    std::vector<uint32_t> lognormal;  // 65537 quantiles of the clipped log-normal length
    std::vector<uint32_t> loguniform; // 65537 quantiles of log-uniform [10k, 1M]
};
const SynthTables& synth_tables();

// ---- BED files (bed.cpp) ------------------------------------------------------------------------
struct BedFile {
    std::string name;                 // file name
    std::vector<std::string> shards;  // in first-appearance order
    std::vector<std::vector<rgl_interval>> ivs;
    uint64_t count = 0;
};
// parse_bed_file (src/io/parse.rs:117-141) of one .bed / .bed.gz file; every interval gets `sid`.
int bed_read(const std::string& path, uint32_t sid, BedFile* f);
// The *.bed / *.bed.gz files of a directory sorted by path, or the path itself.
int bed_list(const std::string& root, std::vector<std::string>* paths, bool* is_dir);
// Parses paths[i] with sid sid0 + i on `threads` threads (0: all cores).
int bed_read_all(const std::vector<std::string>& paths, uint32_t sid0, uint32_t threads, std::vector<BedFile>* out);

// ---- query contexts, for the request server --------------------------------------------------
cudaStream_t context_stream(rgl_context* c);
int context_reserve_rows(rgl_context* c, uint64_t max_intervals, uint32_t max_rows, uint32_t max_blocks);
// Device bytes that running n intervals, `rows` rows and nblk blocks would add to the context's
// workspace (0 when it is already large enough); allocates nothing.
int context_growth_bytes(rgl_context* c, uint64_t n, uint32_t rows, uint32_t nblk, uint64_t* bytes);
// One batch with rows taken from the blocks (interval sids ignored); asynchronous on the context
// stream.  off holds nblk + 1 element offsets into d_iv.
int enqueue_block_rows(rgl_context* c, uint32_t num_rows, uint32_t nblk, const uint32_t* shards, const uint32_t* rows,
                       const uint64_t* off, const rgl_interval* d_iv, const rgl_query_opts* q, uint32_t* d_counts,
                       unsigned long long* d_bp);
// Error bits of the last run, read after the stream has been synchronised.
int context_errors(rgl_context* c);
// The stats stage of rgl_batch_pvalues_device with caller-owned scratch (so that several workers
// can run it at once on one moment store), asynchronous on the context stream unless out_groups.
int batch_pvalues_enqueue(rgl_context* ctx, rgl_moments* m, StatsScratch* sc, const rgl_batch* b,
                          const uint32_t* shard_chrom, uint32_t num_shards, uint32_t bin_size, const uint32_t* d_counts,
                          const uint64_t* d_overlap_bp, double* d_p, double* d_llr, double* d_log_p, uint8_t* d_flags,
                          uint64_t* out_groups);
// Builds the moment store's shared device tables once (thread-safe).
int moments_prepare(rgl_moments* m);
void stats_scratch_release(StatsScratch* sc);
uint32_t context_last_launches(rgl_context* c);

}  // namespace rgl
