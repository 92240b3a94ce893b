"""ctypes binding of libriggle_b200.so (the C ABI declared in include/riggle.h).

The library is built in-tree (``python -m riggle_b200.build``).  Loading fails loudly when it is
missing: there is no CPU fallback for any entry point.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libriggle_b200.so")

RGL_OK = 0
STATUS_NAMES = {
    0: "RGL_OK", 1: "RGL_ERR_INVALID_ARGUMENT", 2: "RGL_ERR_IO", 3: "RGL_ERR_BED_INVALID_FORMAT",
    4: "RGL_ERR_BED_INVALID_START", 5: "RGL_ERR_BED_INVALID_END", 6: "RGL_ERR_BED_INVALID_RANGE",
    7: "RGL_ERR_META_JSON", 8: "RGL_ERR_LAYER_INVALID_POSITION_SIZE", 9: "RGL_ERR_LAYER_INVALID_SID_SIZE",
    10: "RGL_ERR_LAYER_SID_SIZE_MISMATCH", 11: "RGL_ERR_LAYER_INVALID_INDEX_SIZE",
    12: "RGL_ERR_DATABASE_NOT_FOUND", 13: "RGL_ERR_INPUT_NOT_FOUND", 14: "RGL_ERR_NO_BED_FILES",
    15: "RGL_ERR_OOM", 16: "RGL_ERR_TIMEOUT", 17: "RGL_ERR_DEVICE", 18: "RGL_ERR_INDEX_INVARIANT",
    19: "RGL_ERR_NO_DEVICE", 20: "RGL_ERR_UNSUPPORTED",
}
globals().update({v: k for k, v in STATUS_NAMES.items()})


class RiggleError(RuntimeError):
    """A non-zero rgl_status; `.status` holds the code, the message the library's detail."""

    def __init__(self, status, detail):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.name}: {detail}")


class Interval(C.Structure):
    _fields_ = [("start", C.c_uint32), ("end", C.c_uint32), ("sid", C.c_uint32)]


class LayerDesc(C.Structure):
    _fields_ = [("shard", C.c_uint32), ("layer", C.c_uint32), ("count", C.c_uint64),
                ("pos", C.c_void_p), ("sid", C.c_void_p)]


class IndexDesc(C.Structure):
    _fields_ = [("min_size", C.c_uint32), ("growth_factor", C.c_uint32), ("num_sources", C.c_uint32),
                ("num_shards", C.c_uint32), ("shard_names", C.POINTER(C.c_char_p)),
                ("source_names", C.POINTER(C.c_char_p)), ("num_layers", C.c_uint32),
                ("layers", C.POINTER(LayerDesc))]


class IndexInfo(C.Structure):
    _fields_ = [("num_sources", C.c_uint32), ("num_shards", C.c_uint32), ("num_layer_slots", C.c_uint32),
                ("num_layers", C.c_uint32), ("num_intervals", C.c_uint64), ("device_bytes", C.c_uint64),
                ("device", C.c_int)]


class QueryShard(C.Structure):
    _fields_ = [("shard_name", C.c_char_p), ("shard_id", C.c_uint32), ("count", C.c_uint64),
                ("intervals", C.c_void_p)]


class QueryBatch(C.Structure):
    _fields_ = [("num_rows", C.c_uint32), ("num_shards", C.c_uint32), ("shards", C.POINTER(QueryShard))]


class QueryOpts(C.Structure):
    _fields_ = [("chunk", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("block", C.c_uint32), ("flags", C.c_uint32),
                ("pair_ratio", C.c_uint32)]


class QueryStats(C.Structure):
    _fields_ = [("query_intervals", C.c_uint64), ("db_swept", C.c_uint64), ("rank_positions", C.c_uint64),
                ("pair_candidates", C.c_uint64), ("ranges", C.c_uint64),
                ("work_items", C.c_uint64), ("sweep_ms", C.c_float), ("device_ms", C.c_float),
                ("chunk", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("block", C.c_uint32),
                ("kernel_launches", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Pair(C.Structure):
    _fields_ = [("query_start", C.c_uint32), ("query_end", C.c_uint32), ("db_start", C.c_uint32),
                ("db_end", C.c_uint32), ("row", C.c_uint32), ("sid", C.c_uint32), ("shard", C.c_uint32),
                ("intersection_bp", C.c_uint32)]


class BatchDesc(C.Structure):
    _fields_ = [("num_rows", C.c_uint32), ("num_blocks", C.c_uint32), ("block_shards", C.c_void_p),
                ("block_rows", C.c_void_p), ("block_offsets", C.c_void_p), ("d_intervals", C.c_void_p)]


class BatchOpts(C.Structure):
    _fields_ = [("query", QueryOpts), ("sub_batch", C.c_uint64), ("flags", C.c_uint32), ("region_bits", C.c_uint32)]


RGL_BF_GRAPH = 1
RGL_BF_TUNED = 2
RGL_BATCH_NO_REGIONS = 32
RGL_QF_GLOBAL_TALLY = 2


class BatchStats(C.Structure):
    _fields_ = [("query_intervals", C.c_uint64), ("db_swept", C.c_uint64), ("rank_positions", C.c_uint64),
                ("pair_candidates", C.c_uint64), ("ranges", C.c_uint64), ("sub_batches", C.c_uint32),
                ("kernel_launches", C.c_uint32), ("graph_nodes", C.c_uint32), ("graph_replayed", C.c_uint32),
                ("device_ms", C.c_float), ("chunk", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("pair_ratio", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneTrial(C.Structure):
    _fields_ = [("chunk", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("pair_ratio", C.c_uint32),
                ("sweep_ms", C.c_float)]


FREE_MEMORY_FN = C.CFUNCTYPE(C.c_uint64, C.c_void_p)


class ServerOpts(C.Structure):
    _fields_ = [("workers", C.c_uint32), ("max_batch_requests", C.c_uint32), ("batch_intervals", C.c_uint64),
                ("hbm_reserve_bytes", C.c_uint64), ("max_pending_intervals", C.c_uint64), ("query", QueryOpts),
                ("initial_intervals", C.c_uint64), ("free_memory", FREE_MEMORY_FN), ("free_memory_user", C.c_void_p),
                ("moments", C.c_void_p), ("shard_chrom", C.c_void_p), ("num_shard_chrom", C.c_uint32),
                ("bin_size", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("num_blocks", C.c_uint32), ("block_shards", C.c_void_p), ("block_offsets", C.c_void_p),
                ("intervals", C.c_void_p), ("counts", C.c_void_p), ("overlap_bp", C.c_void_p),
                ("p_value", C.c_void_p), ("llr", C.c_void_p), ("log_p", C.c_void_p), ("flags", C.c_void_p)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("batch_requests", C.c_uint32), ("batch_intervals", C.c_uint64),
                ("intervals", C.c_uint64), ("submit_s", C.c_double), ("start_s", C.c_double),
                ("done_s", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("intervals", C.c_uint64), ("workers", C.c_uint32),
                ("pending", C.c_uint32), ("mean_batch_requests", C.c_double), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("p999_ms", C.c_double), ("max_ms", C.c_double), ("mean_ms", C.c_double),
                ("first_submit_s", C.c_double), ("last_done_s", C.c_double), ("worker_bytes", C.c_double),
                ("memory_limited", C.c_uint64), ("refused", C.c_uint64), ("grown_bytes", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SynthSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("num_chroms", C.c_uint32), ("chrom_len", C.POINTER(C.c_uint32)),
                ("num_files", C.c_uint32), ("file_sizes", C.POINTER(C.c_uint64)),
                ("broad_fraction", C.c_double), ("hotspot_fraction", C.c_double),
                ("num_hotspots", C.c_uint32), ("sid_base", C.c_uint32)]


class PValueBatch(C.Structure):
    _fields_ = [("num_rows", C.c_uint32), ("row_group_offsets", C.c_void_p), ("group_chrom", C.c_void_p),
                ("group_l_int", C.c_void_p), ("group_sum_scale", C.c_void_p), ("group_sum_scale2", C.c_void_p),
                ("group_count", C.c_void_p)]


_P = C.c_void_p
_SIGS = {
    "rgl_status_str": (C.c_char_p, [C.c_int]),
    "rgl_last_error": (C.c_char_p, []),
    "rgl_version": (C.c_int, []),
    "rgl_layer_for_size": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "rgl_layer_max_size": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "rgl_tile_size": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "rgl_index_open": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_P)]),
    "rgl_index_open_mem": (C.c_int, [C.POINTER(IndexDesc), C.c_int, C.POINTER(_P)]),
    "rgl_index_close": (C.c_int, [_P]),
    "rgl_index_get_info": (C.c_int, [_P, C.POINTER(IndexInfo)]),
    "rgl_index_shard_id": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_uint32)]),
    "rgl_index_shard_name": (C.c_char_p, [_P, C.c_uint32]),
    "rgl_index_source_name": (C.c_char_p, [_P, C.c_uint32]),
    "rgl_index_layer_count": (C.c_uint64, [_P, C.c_uint32, C.c_uint32]),
    "rgl_index_export_layer": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P]),
    "rgl_context_create": (C.c_int, [_P, _P, C.POINTER(_P)]),
    "rgl_context_destroy": (C.c_int, [_P]),
    "rgl_context_reserve": (C.c_int, [_P, C.c_uint64, C.c_uint32]),
    "rgl_context_stream": (_P, [_P]),
    "rgl_context_sync": (C.c_int, [_P]),
    "rgl_query_counts": (C.c_int, [_P, C.POINTER(QueryBatch), C.POINTER(QueryOpts), _P, _P,
                                   C.POINTER(QueryStats)]),
    "rgl_query_counts_device": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, _P, C.POINTER(QueryOpts), _P, _P,
                                          C.POINTER(QueryStats)]),
    "rgl_query_pairs": (C.c_int, [_P, C.POINTER(QueryBatch), C.c_uint64, _P, C.POINTER(C.c_uint64)]),
    "rgl_query_batch_device": (C.c_int, [_P, C.POINTER(BatchDesc), C.POINTER(BatchOpts), _P, _P,
                                         C.POINTER(BatchStats)]),
    "rgl_query_batch_host": (C.c_int, [_P, C.POINTER(BatchDesc), _P, C.POINTER(BatchOpts), _P, _P,
                                       C.POINTER(BatchStats)]),
    "rgl_batch_autotune": (C.c_int, [_P, C.POINTER(BatchDesc), C.c_uint64, C.POINTER(QueryOpts),
                                     C.POINTER(TuneTrial), C.c_uint32, C.POINTER(C.c_uint32)]),
    "rgl_bed_batch_load": (C.c_int, [C.c_char_p, C.c_uint32, C.POINTER(_P)]),
    "rgl_bed_parse_string": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint32, C.POINTER(_P)]),
    "rgl_bed_batch_rows": (C.c_uint32, [_P]),
    "rgl_bed_batch_row_name": (C.c_char_p, [_P, C.c_uint32]),
    "rgl_bed_batch_row_count": (C.c_uint64, [_P, C.c_uint32]),
    "rgl_bed_batch_row_shards": (C.c_uint32, [_P, C.c_uint32]),
    "rgl_bed_batch_block": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(C.c_char_p), C.POINTER(_P),
                                      C.POINTER(C.c_uint64)]),
    "rgl_bed_batch_query": (C.c_int, [_P, _P, C.POINTER(QueryOpts), _P, _P, C.POINTER(QueryStats)]),
    "rgl_bed_batch_free": (C.c_int, [_P]),
    "rgl_server_create": (C.c_int, [_P, C.POINTER(ServerOpts), C.POINTER(_P)]),
    "rgl_server_submit": (C.c_int, [_P, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "rgl_server_wait": (C.c_int, [_P, C.c_uint64, C.c_uint32, C.POINTER(RequestInfo)]),
    "rgl_server_get_stats": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "rgl_server_reset_stats": (C.c_int, [_P]),
    "rgl_server_destroy": (C.c_int, [_P]),
    "rgl_context_check": (C.c_int, [_P]),
    "rgl_context_set_timing": (C.c_int, [_P, C.c_int]),
    "rgl_context_sweep_times": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_uint32)]),
    "rgl_host_alloc": (C.c_int, [C.c_uint64, C.POINTER(_P)]),
    "rgl_host_free": (C.c_int, [_P]),
    "rgl_compact_index": (C.c_uint64, [C.c_uint64]),
    "rgl_moment_grid": (C.c_uint64, [C.c_uint64, _P, C.c_uint64]),
    "rgl_query_chrom_groups": (C.c_int, [_P, C.c_uint64, C.c_uint32, _P, _P, _P, _P, C.c_uint64,
                                         C.POINTER(C.c_uint64)]),
    "rgl_moments_create": (C.c_int, [C.c_int, C.c_uint32, C.c_uint32, _P, C.POINTER(_P)]),
    "rgl_moments_destroy": (C.c_int, [_P]),
    "rgl_moments_slots": (C.c_uint64, [_P, C.c_uint32]),
    "rgl_moments_set": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, C.c_uint64]),
    "rgl_moments_get": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "rgl_depth_signal": (C.c_int, [C.c_int, _P, C.c_uint64, C.c_uint64, C.c_uint32, _P]),
    "rgl_depth_signal_noalloc": (C.c_int, [C.c_int, _P, C.c_uint64, C.c_uint64, C.c_uint32, _P, _P]),
    "rgl_moments_build": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, C.c_uint64, C.c_uint32, _P, _P]),
    "rgl_moments_build_ex": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, C.c_uint64, C.c_uint32, C.c_uint32, _P, _P]),
    "rgl_query_pvalues": (C.c_int, [_P, C.POINTER(PValueBatch), C.c_uint32, _P, _P, _P, _P, _P, _P]),
    "rgl_batch_pvalues_device": (C.c_int, [_P, _P, C.POINTER(BatchDesc), _P, C.c_uint32, C.c_uint32, _P, _P, _P, _P,
                                           _P, _P, C.POINTER(C.c_uint64)]),
    "rgl_batch_query_groups": (C.c_int, [_P, _P, C.POINTER(BatchDesc), _P, C.c_uint32, C.c_uint32, _P, _P, _P, _P,
                                         _P, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "rgl_synth_chrom_lengths": (C.c_int, [C.c_uint64, C.c_uint32, _P]),
    "rgl_synth_zipf_sizes": (C.c_int, [C.c_uint32, C.c_double, C.c_uint64, C.c_uint64, C.c_uint64, _P]),
    "rgl_synth_loguniform_sizes": (C.c_int, [C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, _P]),
    "rgl_synth_file_chrom_counts": (C.c_int, [C.POINTER(SynthSpec), C.c_uint32, _P]),
    "rgl_synth_block_host": (C.c_int, [C.POINTER(SynthSpec), C.c_uint32, C.c_uint32, _P, C.c_uint64,
                                       C.POINTER(C.c_uint64)]),
    "rgl_synth_chrom_layers_host": (C.c_int, [C.POINTER(SynthSpec), C.c_uint32, C.c_uint32, C.c_uint32, _P,
                                              C.c_uint32, _P, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "rgl_index_synth": (C.c_int, [C.POINTER(SynthSpec), C.c_uint32, C.c_uint32, C.c_int, C.POINTER(_P)]),
    "rgl_index_synth_columns": (C.c_int, [C.POINTER(SynthSpec), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_int, C.POINTER(_P)]),
    "rgl_index_add_beds": (C.c_int, [_P, C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(_P)]),
    "rgl_index_write": (C.c_int, [_P, C.c_char_p]),
    "rgl_index_select_columns": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(_P)]),
    "rgl_synth_batch_layout": (C.c_int, [C.POINTER(SynthSpec), _P, _P, _P]),
    "rgl_synth_batch_device": (C.c_int, [C.POINTER(SynthSpec), C.c_int, _P, _P, _P]),
    "rgl_dense_to_csr_device": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P, _P, C.c_uint64,
                                          C.POINTER(C.c_uint64)]),
    "rgl_format_stats_json": (C.c_int, [C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_uint64,
                                        C.POINTER(C.c_uint64)]),
    "rgl_format_intervals_json": (C.c_int, [_P, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P, _P, _P,
                                            C.c_uint64, C.POINTER(C.c_uint64)]),
    "rgl_abi_struct_name": (C.c_char_p, [C.c_uint32]),
    "rgl_abi_layout": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                 C.POINTER(C.c_char_p), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_uint32]),
}

# The ctypes mirror of every public struct of include/riggle.h, by its C name.
MIRRORS = {
    "rgl_interval": Interval, "rgl_layer_desc": LayerDesc, "rgl_index_desc": IndexDesc,
    "rgl_index_info": IndexInfo, "rgl_query_shard": QueryShard, "rgl_query_batch": QueryBatch,
    "rgl_query_opts": QueryOpts, "rgl_query_stats": QueryStats, "rgl_pair": Pair, "rgl_batch": BatchDesc,
    "rgl_batch_opts": BatchOpts, "rgl_batch_stats": BatchStats, "rgl_tune_trial": TuneTrial,
    "rgl_pvalue_batch": PValueBatch, "rgl_synth_spec": SynthSpec, "rgl_server_opts": ServerOpts,
    "rgl_request": Request, "rgl_request_info": RequestInfo, "rgl_server_stats": ServerStats,
}

EXPORTED = tuple(_SIGS)
_lib = None


def load():
    """Loads the library once; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m riggle_b200.build` "
                               "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status):
    if status != RGL_OK:
        lib = load()
        raise RiggleError(status, lib.rgl_last_error().decode(errors="replace"))
    return status
