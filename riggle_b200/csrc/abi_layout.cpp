// Layout of every public struct of riggle.h as this build of the library sees it, so that a binding
// written in another language (a Rust #[repr(C)] block, Python ctypes) can be checked against the
// compiled ABI instead of against a reading of the header.
#include <cstddef>
#include <cstring>

#include "internal.h"

namespace {

struct FieldRec {
    const char* name;
    uint64_t offset, size;
};
struct StructRec {
    const char* name;
    uint64_t size, align;
    const FieldRec* fields;
    uint32_t num_fields;
};

#define RGL_F(S, f) FieldRec{#f, (uint64_t)offsetof(S, f), (uint64_t)sizeof(((S*)nullptr)->f)}
#define RGL_S(S, arr) StructRec{#S, sizeof(S), alignof(S), arr, (uint32_t)(sizeof(arr) / sizeof(arr[0]))}

const FieldRec f_interval[] = {RGL_F(rgl_interval, start), RGL_F(rgl_interval, end), RGL_F(rgl_interval, sid)};
const FieldRec f_layer_desc[] = {RGL_F(rgl_layer_desc, shard), RGL_F(rgl_layer_desc, layer),
                                 RGL_F(rgl_layer_desc, count), RGL_F(rgl_layer_desc, pos),
                                 RGL_F(rgl_layer_desc, sid)};
const FieldRec f_index_desc[] = {RGL_F(rgl_index_desc, min_size),    RGL_F(rgl_index_desc, growth_factor),
                                 RGL_F(rgl_index_desc, num_sources), RGL_F(rgl_index_desc, num_shards),
                                 RGL_F(rgl_index_desc, shard_names), RGL_F(rgl_index_desc, source_names),
                                 RGL_F(rgl_index_desc, num_layers),  RGL_F(rgl_index_desc, layers)};
const FieldRec f_index_info[] = {RGL_F(rgl_index_info, num_sources),     RGL_F(rgl_index_info, num_shards),
                                 RGL_F(rgl_index_info, num_layer_slots), RGL_F(rgl_index_info, num_layers),
                                 RGL_F(rgl_index_info, num_intervals),   RGL_F(rgl_index_info, device_bytes),
                                 RGL_F(rgl_index_info, device)};
const FieldRec f_query_shard[] = {RGL_F(rgl_query_shard, shard_name), RGL_F(rgl_query_shard, shard_id),
                                  RGL_F(rgl_query_shard, count), RGL_F(rgl_query_shard, intervals)};
const FieldRec f_query_batch[] = {RGL_F(rgl_query_batch, num_rows), RGL_F(rgl_query_batch, num_shards),
                                  RGL_F(rgl_query_batch, shards)};
const FieldRec f_query_opts[] = {RGL_F(rgl_query_opts, chunk), RGL_F(rgl_query_opts, ctas_per_sm),
                                 RGL_F(rgl_query_opts, block), RGL_F(rgl_query_opts, flags),
                                 RGL_F(rgl_query_opts, pair_ratio)};
const FieldRec f_query_stats[] = {RGL_F(rgl_query_stats, query_intervals), RGL_F(rgl_query_stats, db_swept),
                                  RGL_F(rgl_query_stats, rank_positions),  RGL_F(rgl_query_stats, pair_candidates),
                                  RGL_F(rgl_query_stats, ranges),          RGL_F(rgl_query_stats, work_items),
                                  RGL_F(rgl_query_stats, sweep_ms),        RGL_F(rgl_query_stats, device_ms),
                                  RGL_F(rgl_query_stats, chunk),           RGL_F(rgl_query_stats, ctas_per_sm),
                                  RGL_F(rgl_query_stats, block),           RGL_F(rgl_query_stats, kernel_launches)};
const FieldRec f_pair[] = {RGL_F(rgl_pair, query_start), RGL_F(rgl_pair, query_end), RGL_F(rgl_pair, db_start),
                           RGL_F(rgl_pair, db_end),      RGL_F(rgl_pair, row),       RGL_F(rgl_pair, sid),
                           RGL_F(rgl_pair, shard),       RGL_F(rgl_pair, intersection_bp)};
const FieldRec f_batch[] = {RGL_F(rgl_batch, num_rows),   RGL_F(rgl_batch, num_blocks),
                            RGL_F(rgl_batch, block_shards), RGL_F(rgl_batch, block_rows),
                            RGL_F(rgl_batch, block_offsets), RGL_F(rgl_batch, d_intervals)};
const FieldRec f_batch_opts[] = {RGL_F(rgl_batch_opts, query), RGL_F(rgl_batch_opts, sub_batch),
                                 RGL_F(rgl_batch_opts, flags), RGL_F(rgl_batch_opts, region_bits)};
const FieldRec f_batch_stats[] = {RGL_F(rgl_batch_stats, query_intervals), RGL_F(rgl_batch_stats, db_swept),
                                  RGL_F(rgl_batch_stats, rank_positions),  RGL_F(rgl_batch_stats, pair_candidates),
                                  RGL_F(rgl_batch_stats, ranges),          RGL_F(rgl_batch_stats, sub_batches),
                                  RGL_F(rgl_batch_stats, kernel_launches), RGL_F(rgl_batch_stats, graph_nodes),
                                  RGL_F(rgl_batch_stats, graph_replayed),  RGL_F(rgl_batch_stats, device_ms),
                                  RGL_F(rgl_batch_stats, chunk),           RGL_F(rgl_batch_stats, ctas_per_sm),
                                  RGL_F(rgl_batch_stats, pair_ratio)};
const FieldRec f_tune_trial[] = {RGL_F(rgl_tune_trial, chunk), RGL_F(rgl_tune_trial, ctas_per_sm),
                                 RGL_F(rgl_tune_trial, pair_ratio), RGL_F(rgl_tune_trial, sweep_ms)};
const FieldRec f_pvalue_batch[] = {RGL_F(rgl_pvalue_batch, num_rows),        RGL_F(rgl_pvalue_batch, row_group_offsets),
                                   RGL_F(rgl_pvalue_batch, group_chrom),     RGL_F(rgl_pvalue_batch, group_l_int),
                                   RGL_F(rgl_pvalue_batch, group_sum_scale), RGL_F(rgl_pvalue_batch, group_sum_scale2),
                                   RGL_F(rgl_pvalue_batch, group_count)};
const FieldRec f_synth_spec[] = {RGL_F(rgl_synth_spec, seed),           RGL_F(rgl_synth_spec, num_chroms),
                                 RGL_F(rgl_synth_spec, chrom_len),      RGL_F(rgl_synth_spec, num_files),
                                 RGL_F(rgl_synth_spec, file_sizes),     RGL_F(rgl_synth_spec, broad_fraction),
                                 RGL_F(rgl_synth_spec, hotspot_fraction), RGL_F(rgl_synth_spec, num_hotspots),
                                 RGL_F(rgl_synth_spec, sid_base)};
const FieldRec f_server_opts[] = {RGL_F(rgl_server_opts, workers),         RGL_F(rgl_server_opts, max_batch_requests),
                                  RGL_F(rgl_server_opts, batch_intervals), RGL_F(rgl_server_opts, hbm_reserve_bytes),
                                  RGL_F(rgl_server_opts, max_pending_intervals), RGL_F(rgl_server_opts, query),
                                  RGL_F(rgl_server_opts, initial_intervals), RGL_F(rgl_server_opts, free_memory),
                                  RGL_F(rgl_server_opts, free_memory_user), RGL_F(rgl_server_opts, moments),
                                  RGL_F(rgl_server_opts, shard_chrom), RGL_F(rgl_server_opts, num_shard_chrom),
                                  RGL_F(rgl_server_opts, bin_size)};
const FieldRec f_request[] = {RGL_F(rgl_request, num_blocks), RGL_F(rgl_request, block_shards),
                              RGL_F(rgl_request, block_offsets), RGL_F(rgl_request, intervals),
                              RGL_F(rgl_request, counts),     RGL_F(rgl_request, overlap_bp),
                              RGL_F(rgl_request, p_value),    RGL_F(rgl_request, llr),
                              RGL_F(rgl_request, log_p),      RGL_F(rgl_request, flags)};
const FieldRec f_request_info[] = {RGL_F(rgl_request_info, status),          RGL_F(rgl_request_info, batch_requests),
                                   RGL_F(rgl_request_info, batch_intervals), RGL_F(rgl_request_info, intervals),
                                   RGL_F(rgl_request_info, submit_s),        RGL_F(rgl_request_info, start_s),
                                   RGL_F(rgl_request_info, done_s)};
const FieldRec f_server_stats[] = {RGL_F(rgl_server_stats, submitted),      RGL_F(rgl_server_stats, completed),
                                   RGL_F(rgl_server_stats, failed),         RGL_F(rgl_server_stats, batches),
                                   RGL_F(rgl_server_stats, intervals),      RGL_F(rgl_server_stats, workers),
                                   RGL_F(rgl_server_stats, pending),        RGL_F(rgl_server_stats, mean_batch_requests),
                                   RGL_F(rgl_server_stats, p50_ms),         RGL_F(rgl_server_stats, p99_ms),
                                   RGL_F(rgl_server_stats, p999_ms),        RGL_F(rgl_server_stats, max_ms),
                                   RGL_F(rgl_server_stats, mean_ms),        RGL_F(rgl_server_stats, first_submit_s),
                                   RGL_F(rgl_server_stats, last_done_s),    RGL_F(rgl_server_stats, worker_bytes),
                                   RGL_F(rgl_server_stats, memory_limited), RGL_F(rgl_server_stats, refused),
                                   RGL_F(rgl_server_stats, grown_bytes)};

const StructRec g_structs[] = {
    RGL_S(rgl_interval, f_interval),       RGL_S(rgl_layer_desc, f_layer_desc),
    RGL_S(rgl_index_desc, f_index_desc),   RGL_S(rgl_index_info, f_index_info),
    RGL_S(rgl_query_shard, f_query_shard), RGL_S(rgl_query_batch, f_query_batch),
    RGL_S(rgl_query_opts, f_query_opts),   RGL_S(rgl_query_stats, f_query_stats),
    RGL_S(rgl_pair, f_pair),               RGL_S(rgl_batch, f_batch),
    RGL_S(rgl_batch_opts, f_batch_opts),   RGL_S(rgl_batch_stats, f_batch_stats),
    RGL_S(rgl_tune_trial, f_tune_trial),   RGL_S(rgl_pvalue_batch, f_pvalue_batch),
    RGL_S(rgl_synth_spec, f_synth_spec),   RGL_S(rgl_server_opts, f_server_opts),
    RGL_S(rgl_request, f_request),         RGL_S(rgl_request_info, f_request_info),
    RGL_S(rgl_server_stats, f_server_stats),
};
constexpr uint32_t kNumStructs = sizeof(g_structs) / sizeof(g_structs[0]);

}  // namespace

extern "C" {

const char* rgl_abi_struct_name(uint32_t i) { return i < kNumStructs ? g_structs[i].name : nullptr; }

int rgl_abi_layout(const char* name, uint64_t* size, uint64_t* align, uint32_t* num_fields,
                   const char** field_names, uint64_t* offsets, uint64_t* sizes, uint32_t capacity) {
    rgl::clear_error();
    if (!name) return rgl::fail(RGL_ERR_INVALID_ARGUMENT, "struct name is NULL");
    for (const StructRec& s : g_structs) {
        if (std::strcmp(s.name, name) != 0) continue;
        if (size) *size = s.size;
        if (align) *align = s.align;
        if (num_fields) *num_fields = s.num_fields;
        for (uint32_t k = 0; k < s.num_fields && k < capacity; k++) {
            if (field_names) field_names[k] = s.fields[k].name;
            if (offsets) offsets[k] = s.fields[k].offset;
            if (sizes) sizes[k] = s.fields[k].size;
        }
        return RGL_OK;
    }
    return rgl::fail(RGL_ERR_INVALID_ARGUMENT, std::string("no public struct named ") + name);
}

}  // extern "C"
